// Host-side entry points of the MSM pipeline (internal C++ interface below
// the C ABI).
#pragma once

#include "bellman-cuda-b200.h"
#include "msm_kernels.cuh"
#include <cuda_runtime.h>

namespace msm_b200 {

// One MSM request: device or host buffers, any count >= 1.
struct execution {
  cudaMemPool_t pool;
  cudaStream_t stream;
  const void *bases;
  const void *scalars;
  void *results; // 254 Jacobian points
  unsigned count;
  unsigned window_bits; // 0 = default for the size
  cudaEvent_t h2d_event;
  cudaHostFn_t h2d_callback;
  void *h2d_callback_data;
  cudaEvent_t d2h_event;
  cudaHostFn_t d2h_callback;
  void *d2h_callback_data;
  msm_b200_profile *profile;       // optional: synchronous run with stage times and work counts
  const cudaEvent_t *stage_events; // optional: PROFILE_STAGES + 1 caller events recorded at stage boundaries
  unsigned *launches;              // optional: kernels enqueued
};

// windows whose first-pass histograms the digit kernel builds in shared memory
constexpr unsigned MAX_FUSED_HISTOGRAM_WINDOWS = 48;
// Sort tiles below which the unfused path (a digit kernel of one thread per
// point, then histogram + scan + scatter per pass) runs instead: the fused
// digit kernel has one block per tile, too few blocks to fill the GPU.
// Measured on a B200 (plain MSM, default widths): unfused faster up to 2^18
// points (64 tiles; 2^14 at c = 8 0.579 -> 0.466 ms, 2^16 0.683 -> 0.653 ms,
// 2^18 1.217 -> 1.200 ms), fused faster from 2^19 (128 tiles: 1.984 against
// 1.997 ms; 2^20 3.500 against 3.581 ms).
#ifndef FUSED_DIGITS_MIN_TILES
#define FUSED_DIGITS_MIN_TILES 128
#endif

// stages timed by msm_b200_execute_profiled
constexpr unsigned PROFILE_STAGES = 6;

// Accumulation ranges per thread, handed out to warps dynamically.  Measured
// on a B200 at 2^22: 2 per thread cut the plain accumulation from 9.85 to
// 9.32 ms (the last ranges no longer leave SMs idle), 3 gave 9.50 (more heads
// to merge); with the warp-scan head merge, at 2^23, 2 / 3 / 4 per thread
// 18.39 / 18.84 / 18.58 ms.  The batched chain measured best at 1.
#ifndef ACC_RANGES_PER_THREAD
#define ACC_RANGES_PER_THREAD 2
#endif
#ifndef BATCH_ACC_RANGES_PER_THREAD
#define BATCH_ACC_RANGES_PER_THREAD 1
#endif
#ifndef ACC_MIN_RANGE
#define ACC_MIN_RANGE 300 // entries a range keeps at least when ranges are multiplied
#endif

// Per-window sums of the reduction (reduce_groups_kernel, then one
// reduce_level_kernel per level) for the p.windows windows of 2^(c-1) bucket
// slots at `buckets`; afterwards streams[p.log_g & 1] holds each window's sums
// for the gather kernels.  tree / streams: the ping-pong buffers of the plan.
cudaError_t enqueue_window_sums(const plan &p, const xyzz *buckets, const uint8_t *flags, xyzz *const tree[2], xyzz *const streams[2],
                                cudaStream_t stream, unsigned &launched);
// Folds `heads` head partial sums (hb[0], hp[0]; one bucket's heads
// contiguous) into their buckets, level by level, ping-ponging hb / hp.
cudaError_t enqueue_merge_heads(uint32_t *const hb[2], xyzz *const hp[2], unsigned heads, xyzz *buckets, unsigned sms, cudaStream_t stream,
                                unsigned &launched);

unsigned default_window_bits(unsigned long long n);
// Affine pairing levels by size, and a process-wide override (< 0: by size).
constexpr unsigned MAX_AFFINE_LEVELS = 4;
unsigned default_affine_levels(unsigned long long n);
void set_affine_levels_override(int levels);
// p with `levels` affine pairing levels (0 for inputs whose list positions
// would not fit 31 bits), and the geometry of the levels and of the XYZZ pass after them
void set_affine_levels(plan &p, unsigned levels);
// the reduction's groups of 2^log_m bucket slots (capped at the window's slots)
void set_reduction_groups(plan &p, unsigned log_m);
unsigned accumulation_ranges(unsigned threads, unsigned long long entries, unsigned per_thread);
plan make_plan(unsigned n, unsigned window_bits, int sms);
size_t scratch_bytes(unsigned n, unsigned window_bits, bool copy_scalars, bool copy_bases, bool copy_results);
cudaError_t execute(const execution &e);
cudaError_t set_up();

} // namespace msm_b200
