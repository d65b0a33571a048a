/*
 * bellman-cuda.h -- C ABI of the B200 BN254 G1 MSM library.
 *
 * This is a drop-in for the MSM part of era-bellman-cuda's public header
 * (src/bellman-cuda.h in that project): the same type names, enum values,
 * struct layouts and function signatures, so a prover compiled against the
 * reference header links against this library unchanged.  Each declaration
 * below names the reference declaration it replaces.
 *
 * Exported: the bc_* runtime wrappers, ff_set_up / ff_tear_down (accepted and
 * validated; the MSM does not use field twiddle tables) and
 * msm_set_up / msm_execute_async / msm_tear_down.  The reference's NTT,
 * vector field-operation and permutation-polynomial entry points are not part
 * of this library.
 *
 * Error codes are the CUDA runtime codes of the failing call, exactly as the
 * reference returns them (its wrappers static_cast every cudaError_t).
 */
#pragma once

#ifndef __cplusplus
#include <stdbool.h>
#include <stddef.h>
#else
#include <cstddef>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default) /* the library builds with hidden visibility */
#endif

/* reference: src/bellman-cuda.h:13-21 (values equal the CUDA runtime codes) */
typedef enum bc_error {
  bc_success = 0,
  bc_error_invalid_value = 1,
  bc_error_memory_allocation = 2,
  bc_error_not_ready = 600
} bc_error;

/* reference: src/bellman-cuda.h:24-36 -- opaque handles wrapping cudaStream_t,
 * cudaEvent_t and cudaMemPool_t */
typedef struct bc_stream {
  void *handle;
} bc_stream;

typedef struct bc_event {
  void *handle;
} bc_event;

typedef struct bc_mem_pool {
  void *handle;
} bc_mem_pool;

/* reference: src/bellman-cuda.h:40 */
typedef void (*bc_host_fn)(void *user_data);

/* ---- devices (reference: src/bellman-cuda.h:44-52) ---------------------- */
bc_error bc_get_device_count(int *count);
bc_error bc_get_device(int *device_id);
bc_error bc_set_device(int device_id);

/* ---- streams (reference: src/bellman-cuda.h:57-81) ----------------------- */
/* blocking_sync: the stream waits with a blocking primitive instead of spinning */
bc_error bc_stream_create(bc_stream *stream, bool blocking_sync);
bc_error bc_stream_wait_event(bc_stream stream, bc_event event);
bc_error bc_stream_synchronize(bc_stream stream);
/* bc_success when all work is done, bc_error_not_ready otherwise */
bc_error bc_stream_query(bc_stream stream);
bc_error bc_stream_destroy(bc_stream stream);
bc_error bc_launch_host_fn(bc_stream stream, bc_host_fn fn, void *user_data);

/* ---- events (reference: src/bellman-cuda.h:87-111) ------------------------ */
bc_error bc_event_create(bc_event *event, bool blocking_sync, bool disable_timing);
bc_error bc_event_record(bc_event event, bc_stream stream);
bc_error bc_event_synchronize(bc_event event);
bc_error bc_event_query(bc_event event);
bc_error bc_event_destroy(bc_event event);
bc_error bc_event_elapsed_time(float *ms, bc_event start, bc_event end);

/* ---- memory (reference: src/bellman-cuda.h:116-208) ----------------------- */
bc_error bc_mem_get_info(size_t *free, size_t *total);
bc_error bc_malloc(void **ptr, size_t size);
bc_error bc_malloc_host(void **ptr, size_t size);
bc_error bc_free(void *ptr);
bc_error bc_free_host(void *ptr);
bc_error bc_host_register(void *ptr, size_t size);
bc_error bc_host_unregister(void *ptr);
bc_error bc_device_disable_peer_access(int device_id);
bc_error bc_device_enable_peer_access(int device_id);
bc_error bc_memcpy(void *dst, const void *src, size_t count);
bc_error bc_memcpy_async(void *dst, const void *src, size_t count, bc_stream stream);
bc_error bc_memset(void *ptr, int value, size_t count);
bc_error bc_memset_async(void *ptr, int value, size_t count, bc_stream stream);
/* a device memory pool whose release threshold is unbounded, so memory freed
 * back to it is kept for the next MSM */
bc_error bc_mem_pool_create(bc_mem_pool *pool, int device_id);
bc_error bc_mem_pool_destroy(bc_mem_pool pool);
bc_error bc_mem_pool_disable_peer_access(bc_mem_pool pool, int device_id);
bc_error bc_mem_pool_enable_peer_access(bc_mem_pool pool, int device_id);
bc_error bc_malloc_from_pool_async(void **ptr, size_t size, bc_mem_pool pool, bc_stream stream);
bc_error bc_free_async(void *ptr, bc_stream stream);

/* ---- field set-up (reference: src/bellman-cuda.h:214, :431) ---------------
 * Accepted for ABI compatibility; both counts must be <= 28 (the 2-adicity of
 * the scalar field).  The MSM needs no field tables. */
bc_error ff_set_up(unsigned powers_of_w_coarse_log_count, unsigned powers_of_g_coarse_log_count);
bc_error ff_tear_down();

/* ---- MSM (reference: src/bellman-cuda.h:474-509) --------------------------- */

/* Once per process and device: kernel attributes. */
bc_error msm_set_up();

/* reference: src/bellman-cuda.h:477-491, same field order and types */
typedef struct msm_configuration {
  bc_mem_pool mem_pool;                  /* pool for all temporary allocations (stream-ordered on `stream`) */
  bc_stream stream;                      /* stream the MSM is enqueued on */
  void *bases;                           /* 2^log_scalars_count affine points (x, y), Montgomery-form Fq, 64 B each, 16 B aligned */
  void *scalars;                         /* 2^log_scalars_count Montgomery-form Fr scalars, 32 B each; device, pinned or pageable */
  void *results;                         /* 254 Jacobian points (x, y, z), Montgomery-form Fq, 96 B each; device, pinned or pageable */
  unsigned log_scalars_count;            /* log2 of the number of points */
  bc_event h2d_copy_finished;            /* optional: recorded once host inputs have been copied to the device */
  bc_host_fn h2d_copy_finished_callback; /* optional: called at the same point */
  void *h2d_copy_finished_callback_data;
  bc_event d2h_copy_finished;            /* optional: recorded once host results have been written */
  bc_host_fn d2h_copy_finished_callback; /* optional: called at the same point */
  void *d2h_copy_finished_callback_data;
} msm_configuration;

/*
 * Enqueue sum_i scalars[i] * bases[i] on configuration.stream.
 *
 * The result is delivered as 254 points R_0..R_253 with
 *     MSM = sum_i 2^i * R_i,
 * which the caller reduces, e.g. by Horner from the top:
 *     sum = R_253;  for i = 252 .. 0:  sum = 2 * sum + R_i.
 * Only that sum is defined: the individual R_i depend on the window split.
 * Jacobian infinity is (0, 1, 0) in Montgomery form.
 *
 * Scratch comes from configuration.mem_pool in stream order.  When the pool
 * cannot hold the scratch of the whole MSM, the points are processed in
 * smaller equal chunks (halved until they fit, down to 2^16 points), as the
 * reference's dry-run fit does (src/msm.cu:431-459); bc_error_memory_allocation
 * only when even that does not fit.  Device memory of another device is
 * refused (bc_error_invalid_value) unless peer access to it was enabled
 * through bc_device_enable_peer_access.
 */
bc_error msm_execute_async(msm_configuration configuration);

bc_error msm_tear_down();

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
} /* extern "C" */
#endif
