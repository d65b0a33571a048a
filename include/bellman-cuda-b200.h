/*
 * bellman-cuda-b200.h -- extensions of the B200 MSM library beyond the
 * era-bellman-cuda ABI (which is declared, unchanged, in bellman-cuda.h).
 * None of these has a counterpart in the reference.
 */
#pragma once

#include "bellman-cuda.h"
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default) /* the library builds with hidden visibility */
#endif

/* An MSM of any length (the reference's msm_execute_async takes powers of two
 * only).  Same buffers and result convention as msm_execute_async. */
typedef struct msm_b200_configuration {
  bc_mem_pool mem_pool; /* may be a null handle: the device's default pool */
  bc_stream stream;
  const void *bases;    /* count affine points, Montgomery form, 64 B each */
  const void *scalars;  /* count Montgomery-form scalars, 32 B each */
  void *results;        /* 254 Jacobian points, MSM = sum_i 2^i R_i */
  unsigned count;       /* >= 1 */
  unsigned window_bits; /* 0: size-based default; otherwise 2..24 */
} msm_b200_configuration;

bc_error msm_b200_execute_async(const msm_b200_configuration *configuration);

/* Per-stage device times and work counts of one MSM. */
typedef struct msm_b200_profile {
  float stage_ms[6];                   /* digits, sort, zero counts, accumulation, head merge, bucket reduction */
  unsigned long long nonzero_entries;  /* (window, point) pairs with a nonzero digit */
  unsigned long long nonempty_buckets; /* buckets that received at least one point */
  unsigned long long heads;            /* accumulation ranges that began inside a bucket */
  unsigned window_bits, windows, acc_threads /* accumulation ranges */, launches;
  unsigned sort_wait_timeouts; /* radix-pass look-back waits that gave up (0 in correct operation) */
  unsigned affine_levels;                /* affine pairing levels run before the XYZZ accumulation */
  unsigned long long affine_additions;   /* list elements those levels removed (one per affine pair sum) */
} msm_b200_profile;

/* Same as msm_b200_execute_async, but synchronises the stream before it
 * returns and fills *profile.  Mixed (XYZZ += affine) additions performed by
 * the accumulation = nonzero_entries - affine_additions - nonempty_buckets -
 * heads. */
bc_error msm_b200_execute_profiled(const msm_b200_configuration *configuration, msm_b200_profile *profile);

/* Affine pairing levels of later plain MSMs (msm_execute_async and the
 * msm_b200_execute_* calls; the batched path and the server do not use
 * them), process-wide: 0..4 levels for every size, or a negative value for
 * the default (none).  Each level adds, in
 * affine coordinates, every two consecutive sorted entries of one bucket, all
 * of a level's slopes sharing one field inversion (5 products and 1 square per
 * addition against the XYZZ madd's 8 and 2); the XYZZ accumulation then adds
 * what is left.  Results are the same group elements either way.  On a B200
 * the levels measure slower than the XYZZ pass at every size (each level
 * streams its list through memory twice, and the first gathers every base
 * twice), hence the default. */
bc_error msm_b200_set_affine_levels(int levels);

/* msm_b200_execute_async that also records stage_events[0..6] on the stream:
 * before the first stage and after each of the six stages of
 * msm_b200_profile.stage_ms (no synchronisation).  *launches (optional)
 * receives the number of kernels enqueued. */
bc_error msm_b200_execute_staged_async(const msm_b200_configuration *configuration, const bc_event *stage_events, unsigned *launches);

/* Throughput of 32-bit multiply instructions on the current device, in
 * multiply instructions per second (mul.lo / mul.hi / mad* each count one):
 *   kind 0: independent mad.lo / mad.hi (the integer multiply pipe's peak)
 *   kind 1: carry chains of madc.lo.cc / madc.hi.cc pairs
 *   kind 2: Fq Montgomery products (264 multiply instructions each)
 *   kind 3: XYZZ + affine mixed additions (2392 multiply instructions each)
 *   kind 4: independent mad.lo only
 * Synchronous; about 0.1 s. */
bc_error msm_b200_measure_mul_throughput(unsigned kind, double *mulops_per_second);

/* Bytes of pool memory one device-resident MSM of `count` points takes. */
bc_error msm_b200_scratch_bytes(unsigned count, unsigned window_bits, size_t *bytes);

/* The window width msm_execute_async uses for `count` points. */
bc_error msm_b200_default_window_bits(unsigned count, unsigned *window_bits);

/* bases[i] = k[i] * G for the generator G = (1, 2), as Montgomery-form affine
 * points (64 B each).  k: `count` standard-form scalars in [1, r), device
 * memory.  Used to build synthetic base tables on the device. */
bc_error msm_b200_generator_multiples_async(const void *k, void *bases, unsigned count, bc_stream stream);

/* ---- Batched MSMs over one resident base table (no counterpart in the
 * reference).
 *
 * A base table keeps `count` affine points (Montgomery form, 64 B each) on the
 * device together with their precomputed window multiples 2^(c j) P_i for one
 * or more window widths c, so that an MSM over a prefix of the table needs a
 * single set of 2^(c-1) buckets.  A batch is a fixed list of instance lengths
 * (each a prefix of the table); all its instances run as one kernel chain over
 * a shared work list, captured once in a CUDA graph and replayed by every
 * execution.  Results follow the msm_execute_async convention (254 Jacobian
 * points per instance, MSM = sum_i 2^i R_i; here R_i = 0 for i >= c). */
#define MSM_B200_MAX_BATCH 256u
typedef struct msm_b200_base_table_t *msm_b200_base_table;
typedef struct msm_b200_batch_t *msm_b200_batch;

/* Builds a table from `bases` (device or host memory; copied).  window_bits:
 * the widths to precompute (widths entries, 2..24); with widths = 0 the widths
 * msm_b200_batch_window_bits picks for every length up to `count`, each only
 * for the prefix that lengths of that width can reach.  Synchronous on
 * `stream`; the table owns its device memory until destroyed. */
bc_error msm_b200_base_table_create(msm_b200_base_table *table, const void *bases, unsigned count, const unsigned *window_bits, unsigned widths,
                                    bc_stream stream);
/* Device bytes the table holds. */
bc_error msm_b200_base_table_bytes(msm_b200_base_table table, size_t *bytes);
bc_error msm_b200_base_table_destroy(msm_b200_base_table table);
/* Save / load format of a table: a little-endian header (the words
 * 0x34354e42 0x4c424154, version 1, point count, number of widths, then per
 * width c, prefix, windows) followed by each width's windows x prefix affine
 * points (Montgomery form, 64 B each), widths in increasing order.  Export
 * writes it into host memory of msm_b200_base_table_serialized_bytes bytes
 * (synchronous); import rebuilds the table on the current device without
 * recomputing the multiples and rejects a malformed or truncated image with
 * bc_error_invalid_value. */
bc_error msm_b200_base_table_serialized_bytes(msm_b200_base_table table, size_t *bytes);
bc_error msm_b200_base_table_export(msm_b200_base_table table, void *image, size_t bytes);
bc_error msm_b200_base_table_import(msm_b200_base_table *table, const void *image, size_t bytes, bc_stream stream);

/* The window width the batched path uses for an instance of `count` points:
 * the checked-in table written by the autotuner (era-bellman-cuda_b200/autotune.py). */
bc_error msm_b200_batch_window_bits(unsigned count, unsigned *window_bits);

/* Plans a batch of `instances` (1..MSM_B200_MAX_BATCH) MSMs of counts[k]
 * points over the first counts[k] points of `table`; window_bits (optional, 0
 * entries = tuned) forces per-instance widths, which the table must hold.
 * Allocates the batch's scratch (cudaMalloc) and captures its CUDA graph. */
bc_error msm_b200_batch_create(msm_b200_batch *batch, msm_b200_base_table table, const unsigned *counts, unsigned instances,
                               const unsigned *window_bits);
/* Runs the batch: scalars[k] (counts[k] Montgomery-form scalars) and
 * results[k] (254 Jacobian points) are device pointers.  Executions of one
 * batch share its scratch: serialise them (one stream). */
bc_error msm_b200_batch_execute_async(msm_b200_batch batch, const void *const *scalars, void *const *results, bc_stream stream);
/* Scratch bytes, kernels in the graph, and (window, point) entries of a batch
 * (each window padded to a whole number of 4096-point sort tiles). */
bc_error msm_b200_batch_info(msm_b200_batch batch, size_t *scratch_bytes, unsigned *kernels, unsigned long long *entries);
bc_error msm_b200_batch_destroy(msm_b200_batch batch);

/* ---- Request server (no counterpart in the reference): continuous batching
 * of MSM requests over one resident base table.
 *
 * Requests are submitted from any thread and queue in arrival order.  A
 * scheduler thread admits them, oldest first, into groups that run as one
 * batched kernel chain on one of `streams` device streams: a group grows
 * while its scratch footprint fits in the largest free block of a device arena
 * of `scratch_budget` bytes (allocated once, at creation) and it has at most
 * `max_group` requests.  Groups admitted while others are still running
 * overlap with them on the device; a finished group frees its arena block and
 * stream, which admits the next requests.  A request longer than the table, or
 * whose footprint exceeds the whole arena, finishes with an error. */
typedef struct msm_b200_server_t *msm_b200_server;

/* Host clock (microseconds since the server was created) of one request. */
typedef struct msm_b200_request_times {
  double submit_us, start_us, done_us; /* submitted, its group enqueued, its group finished */
  unsigned group_size;                 /* requests in its group */
} msm_b200_request_times;

typedef struct msm_b200_server_stats {
  unsigned long long groups, requests, max_inflight_groups;
  size_t arena_bytes, arena_used, pending;
} msm_b200_server_stats;

bc_error msm_b200_server_create(msm_b200_server *server, msm_b200_base_table table, size_t scratch_budget, unsigned streams, unsigned max_group);
/* Queues an MSM of `count` points over the first `count` points of the table.
 * scalars: count Montgomery-form scalars; results: 254 Jacobian points (as
 * msm_execute_async); each in device or host memory (host scalars are copied
 * in when the request starts; pinned memory keeps the scheduler from
 * blocking), valid until msm_b200_server_wait returns for the ticket. */
bc_error msm_b200_server_submit(msm_b200_server server, const void *scalars, unsigned count, void *results, unsigned long long *ticket);
/* Blocks until the request has finished; returns its status and (optional)
 * its times, then forgets the ticket. */
bc_error msm_b200_server_wait(msm_b200_server server, unsigned long long ticket, msm_b200_request_times *times);
bc_error msm_b200_server_get_stats(msm_b200_server server, msm_b200_server_stats *stats);
/* Finishes the queued requests, then releases the arena and streams. */
bc_error msm_b200_server_destroy(msm_b200_server server);

/* An MSM that allocates no memory (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory at call time: code running
 * inside a host callback or a driver/loader layer where cudaMalloc is not
 * allowed, a prover whose device memory is pre-committed by its own
 * allocator, or a process that must not grow its footprint after start-up.
 * Every other MSM entry point takes its scratch from a memory pool on every
 * call; this one uses a fixed block of device memory that is part of the
 * library image (MSM_B200_NO_ALLOC_SCRATCH_BYTES, 64 MiB), which every GPU
 * that loads the library holds until the process exits.
 *
 * bases, scalars and results must all be device memory (nothing is copied
 * in or out); layout and result convention as msm_execute_async, with any
 * count in [1, MSM_B200_NO_ALLOC_MAX_COUNT].  A count outside that range, a
 * null or host pointer, or a misaligned buffer returns bc_error_invalid_value
 * before anything is enqueued.  The window width is the size-based default.
 *
 * The first call in a CUDA context looks up the block's device address in
 * that context (cudaGetSymbolAddress, cached by the context's unique id, so a
 * device reset or a caller's own context gets a fresh lookup); make that
 * first call before any stream capture.  Device memory of another device is
 * refused unless peer access to it was enabled through
 * bc_device_enable_peer_access.  Every call shares the one block and the block keeps the last
 * call's contents (whatever must start at zero is cleared by each call): two
 * calls whose work overlaps on the GPU, on different streams or from
 * different threads, race and both results are undefined.  Serialise them,
 * e.g. on one stream. */
#define MSM_B200_NO_ALLOC_MAX_COUNT 65536u
#define MSM_B200_NO_ALLOC_SCRATCH_BYTES (64u << 20)
bc_error msm_b200_execute_no_alloc_async(bc_stream stream, const void *bases, const void *scalars, void *results, unsigned count);

/* The caller-side final reduction on the GPU (no counterpart in the
 * reference, whose callers run it on the host: src/bellman-cuda.h:496-505).
 *
 * Writes sum over i < 254 of 2^i R_i of the 254 Jacobian points at `results`
 * (the layout msm_execute_async writes: Montgomery-form Fq coordinates below
 * 2p, x = X/Z^2, y = Y/Z^3, Z = 0 for infinity; this library's results and
 * the reference's both qualify) to `point` as one canonical affine point:
 * x and y in standard (not Montgomery) form, fully reduced mod p, 8
 * little-endian 32-bit limbs each; infinity = 1 and x = y = 0 for the point
 * at infinity.  The bytes therefore compare equal for equal points, whatever
 * window split produced the R_i.
 *
 * `results` (16-byte aligned) and `point` must be device memory of the
 * current device, device memory of another device to which the current one
 * has peer access enabled through bc_device_enable_peer_access, managed
 * memory, or pinned host memory (registered or cudaMallocHost'd; the kernel
 * reads and writes it in place); a null or pageable pointer, or another
 * device's memory without that peer access, returns bc_error_invalid_value
 * before anything is enqueued.  Asynchronous on `stream`, one kernel of one block, no
 * allocation.  Enqueue it after the MSM on the same stream.
 *
 * Speed: this is not a faster Horner pass.  The sum needs 253 doublings in a
 * dependent chain whatever the order, and one GPU thread's carry chains are
 * slower than a host core's 64-bit products: about 0.55 ms per call on a B200
 * for this library's plain results, against about 0.21 ms for the Horner
 * pass on one host core of the same machine (0.13 ms here for batched
 * results, whose upper bits are infinity).  Use it when the point is wanted
 * on the device, or when the host should do no work; otherwise the host pass
 * is quicker. */
typedef struct msm_b200_affine_point {
  uint32_t x[8];
  uint32_t y[8];
  uint32_t infinity;
  uint32_t reserved[3];
} msm_b200_affine_point;
bc_error msm_b200_final_sum_async(const void *results, msm_b200_affine_point *point, bc_stream stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
} /* extern "C" */
#endif
