// Device kernels of the Pippenger MSM pipeline (one GPU, sm_100a).
//
// Pipeline for n points, window width c, W = ceil(254 / c) windows and
// B = 2^(c-1) bucket slots per window:
//   1. digits      scalars -> signed c-bit digits of min(s, r - s); per window
//                  a key |d| - 1 (c - 1 bits; a zero digit wraps to ZERO_KEY)
//                  and a value (point index | sign << 31)
//   2. sort        LSD radix sort of (key, value) inside each window segment;
//                  the first pass drops zero digits (counted per window), so
//                  window w keeps its nonzero entries at the end of its segment
//   4. accumulate  the nonzero entries of all windows are split into equal
//                  contiguous ranges, handed out to warps; each thread adds its
//                  range bucket by bucket (XYZZ += affine); buckets that start
//                  inside a range are written directly, a bucket continued
//                  from the previous range leaves a "head" partial sum
//                  (optionally preceded by affine pairing levels, off by
//                  default: msm_affine.cuh)
//   5. merge_heads heads of one bucket are contiguous; a segmented scan of 32
//                  heads per warp, repeated until every head is folded into
//                  its bucket
//   6. reduction   per window S_w = sum_k k * X_k (X_k = bucket of |d| = k,
//                  slot 0 holds |d| = B): running sums over groups of m slots,
//                  then a binary decomposition of the group weights, so every
//                  partial result is a plain sum placed at the bit position it
//                  belongs to in the 254-entry result array.
// The caller's Horner pass over the 254 results (sum 2^i R_i) completes the
// MSM, exactly as with the reference (src/bellman-cuda.h:496-505).
#pragma once

#include "bn254_curve.cuh"
#include <cuda_runtime.h>

namespace msm_b200 {

using bn254::affine;
using bn254::curve;
using bn254::fe;
using bn254::fq;
using bn254::fr;
using bn254::jacobian;
using bn254::xyzz;

constexpr unsigned RESULT_BITS = 254;
constexpr unsigned INVALID_BUCKET = 0xffffffffu;
constexpr unsigned SORT_RADIX_BITS = 8;
constexpr unsigned SORT_RADIX = 1u << SORT_RADIX_BITS;
constexpr unsigned SORT_THREADS = 256;
constexpr unsigned SORT_ITEMS = 16; // per thread; a tile is SORT_THREADS * SORT_ITEMS keys
constexpr unsigned SORT_TILE = SORT_THREADS * SORT_ITEMS;
// Resident scatter blocks per SM (4 caps registers at 64, with a few bytes of
// spills): at 2^22 the sort stage took 1.067 ms at 3 blocks, 1.012 at 4.
// Resident blocks per SM the reduction kernels are compiled for (1: as many
// as their registers allow).  reduce_groups_kernel at 3 (168 registers, 140
// bytes of spills, instead of 206 registers and 2 blocks): reduction stage at
// 2^22 0.695 -> 0.664 ms with groups of 8 slots, 0.692 -> 0.637 ms with the
// groups of 4 it uses there now; reduce_level_kernel at 4 measured no better.
#ifndef REDUCE_GROUPS_MIN_BLOCKS
#define REDUCE_GROUPS_MIN_BLOCKS 3
#endif
#ifndef REDUCE_LEVEL_MIN_BLOCKS
#define REDUCE_LEVEL_MIN_BLOCKS 1
#endif
#ifndef SORT_SCATTER_MIN_BLOCKS
#define SORT_SCATTER_MIN_BLOCKS 4
#endif
// The look-back passes (the radix passes after the first): blocks of 256
// threads with 16 items each, the sort tiles of the first pass.  Measured on
// a B200 at 2^22 (c = 17, sort stage of the plain MSM, scan + first pass +
// one look-back pass): 0.803 ms with these tiles, 0.822 with blocks of 512
// threads x 12 items (tiles of 6144, 2 blocks per SM), 0.832 with the
// earlier look-back over separate flag and count arrays.  (A standalone pass
// over the same sizes favoured the larger tiles, 0.410 against 0.439 ms; in
// the pipeline the gain did not hold.)
constexpr unsigned LOOKBACK_THREADS = SORT_THREADS, LOOKBACK_ITEMS = SORT_ITEMS, LOOKBACK_TILE = LOOKBACK_THREADS * LOOKBACK_ITEMS;
// Dynamic shared memory of a look-back tile of THREADS x ITEMS entries: the
// staged tile (key and value in one 8-byte word) and per-warp digit counters.
template <unsigned THREADS, unsigned ITEMS> constexpr size_t lookback_smem_bytes() {
  return (size_t)THREADS * ITEMS * 8 + (size_t)(THREADS / 32) * SORT_RADIX * 4;
}
constexpr unsigned ACC_THREADS = 128;

// Window w's entries start at w * window_stride(n): n rounded up to 32
// entries, so that every window segment starts on a 128-byte line and the
// digit kernels' stores stay whole lines whatever n is (at n = 3,495,254
// the digit stage took 0.220 ms, at the aligned 3,495,264 0.141 ms).
__host__ __device__ __forceinline__ size_t window_stride(unsigned n) { return ((size_t)n + 31) & ~(size_t)31; }

// Launch geometry of the whole pipeline, computed on the host.
struct plan {
  unsigned n;           // points
  unsigned c;           // window bits
  unsigned windows;     // W
  unsigned log_b;       // log2 of bucket slots per window (c - 1)
  unsigned key_bits;    // bits of a sort key (|d| - 1 for |d| in [1, 2^log_b])
  unsigned sort_passes; // radix passes
  unsigned tiles;       // sort tiles per window
  unsigned lookback_tiles; // look-back tiles (LOOKBACK_TILE entries) per window
  unsigned acc_threads; // accumulation threads (4 blocks of ACC_THREADS per SM at most)
  unsigned acc_ranges;  // accumulation ranges (>= acc_threads), handed out to warps
  unsigned log_m;       // log2 of the running-sum group
  unsigned groups;      // G = B / m groups per window
  unsigned log_g;       // gamma = log2 G
  unsigned sms;         // SMs of the device the plan is for
  unsigned affine_levels; // affine pairing levels before the XYZZ accumulation (0: none)
  unsigned level_warps;   // warps of each level's grid
  unsigned tail_threads;  // XYZZ accumulation threads and ranges after the levels
  unsigned tail_ranges;
};

// ---------------------------------------------------------------------------
// 1. digits
// ---------------------------------------------------------------------------
// Signed windows of s' = min(s, r - s) < 2^253 (reference fold,
// src/msm_kernels.cu:49-52): raw = bits [c*w, c*w + c) + carry; a raw value
// above B becomes raw - 2^c with a carry into the next window.  |d| <= B,
// and the top window of a W*c >= 254 split never carries out.
__global__ void digits_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows, uint32_t *__restrict__ keys,
                              uint32_t *__restrict__ vals);
// the same, one block per sort tile, also counting the tile's nonzero keys
// per window and radix digit for every sort pass and adding each window's
// zero digits to zeros[w]
__global__ void digits_histogram_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows, unsigned passes, unsigned tiles,
                                        uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, uint32_t *__restrict__ hist,
                                        uint32_t *__restrict__ totals, uint32_t *__restrict__ zeros);
// a stable radix pass in one kernel, positions by decoupled look-back
// (tiles: look-back tiles per window; words: [windows][tiles][256], zero at
// launch; dynamic shared memory lookback_smem_bytes<LOOKBACK_THREADS,
// LOOKBACK_ITEMS>())
__global__ void lookback_stable_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                                       uint32_t *__restrict__ vals_out, unsigned n, unsigned windows, unsigned tiles, unsigned shift, uint32_t *words,
                                       const uint32_t *__restrict__ totals, const uint32_t *__restrict__ zeros, unsigned *tile_ctr, unsigned *error);

// ---------------------------------------------------------------------------
// 2. sort (keys and values per window segment of n entries); the first pass
//    drops zero digits, counting them in zeros[w] (which must start at 0)
// ---------------------------------------------------------------------------
__global__ void sort_histogram_first_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles, unsigned shift,
                                            uint32_t *__restrict__ counts, uint32_t *__restrict__ zeros);
__global__ void sort_histogram_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles, unsigned shift, uint32_t *__restrict__ counts,
                                      const uint32_t *__restrict__ zeros);
__global__ void sort_scan_kernel(uint32_t *counts, unsigned tiles, unsigned rows, uint32_t *__restrict__ totals);
// first pass (any order among equal digits) and later passes (stable)
__global__ void sort_scatter_first_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                                          uint32_t *__restrict__ vals_out, unsigned n, unsigned tiles, unsigned shift,
                                          const uint32_t *__restrict__ counts, const uint32_t *__restrict__ totals,
                                          const uint32_t *__restrict__ zeros);
__global__ void sort_scatter_stable_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                                           uint32_t *__restrict__ vals_out, unsigned n, unsigned tiles, unsigned shift,
                                           const uint32_t *__restrict__ counts, const uint32_t *__restrict__ totals,
                                           const uint32_t *__restrict__ zeros);

// ---------------------------------------------------------------------------
// 4. accumulation
// ---------------------------------------------------------------------------
// `ranges` equal ranges handed out to warps through *work (0 at launch)
__global__ void accumulate_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, const affine *__restrict__ bases,
                                  unsigned n, unsigned windows, unsigned log_b, const uint32_t *__restrict__ zeros, unsigned ranges,
                                  unsigned *__restrict__ work, xyzz *__restrict__ buckets, uint8_t *__restrict__ flags,
                                  uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point);

// Affine pairing levels ahead of the accumulation (msm_affine.cuh).
constexpr unsigned AFFINE_FORWARD_THREADS = 256;
constexpr unsigned AFFINE_APPLY_THREADS = 128;
constexpr unsigned AFFINE_INVERT_THREADS = 512;
#ifndef AFFINE_APPLY_MIN_BLOCKS
#define AFFINE_APPLY_MIN_BLOCKS 4 // resident apply blocks per SM (caps registers at 128)
#endif
// Per-level arrays of a grid of `warps` warps:
struct level_arrays {
  fe *pre;                       // per pair: product of the lane's earlier slope denominators
  fe *others;                    // per lane: product of the other lanes' chain totals
  fe *warp_total;                // per warp: product of all its slope denominators
  fe *warp_inverse;              // per warp: inverse of warp_total
  uint32_t *warp_outputs;        // per warp: output elements
  unsigned long long *warp_base; // per warp: position of its first output element
  unsigned long long *count_out; // output elements of the level
  uint32_t *out_buckets;         // output list: global bucket ids and points
  affine *out_points;
};
// level 1 over the sorted nonzero entries of the windows (as accumulate_kernel reads them)
__global__ void affine_forward_first_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, const affine *__restrict__ bases,
                                            unsigned n, unsigned windows, unsigned log_b, const uint32_t *__restrict__ zeros, level_arrays a,
                                            unsigned warps);
__global__ void affine_apply_first_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, const affine *__restrict__ bases,
                                          unsigned n, unsigned windows, unsigned log_b, const uint32_t *__restrict__ zeros, level_arrays a,
                                          unsigned warps);
// later levels over the previous level's list of *count elements
__global__ void affine_forward_list_kernel(const uint32_t *__restrict__ list_buckets, const affine *__restrict__ points,
                                           const unsigned long long *__restrict__ count, level_arrays a, unsigned warps);
__global__ void affine_apply_list_kernel(const uint32_t *__restrict__ list_buckets, const affine *__restrict__ points,
                                         const unsigned long long *__restrict__ count, level_arrays a, unsigned warps);
// one block: warp_inverse, warp_base and *count_out of a level
__global__ void affine_invert_kernel(const fe *__restrict__ warp_total, const uint32_t *__restrict__ warp_outputs, unsigned warps,
                                     fe *__restrict__ warp_inverse, unsigned long long *__restrict__ warp_base,
                                     unsigned long long *__restrict__ count_out);
// the XYZZ accumulation over the last level's list of *count elements
__global__ void accumulate_list_kernel(const uint32_t *__restrict__ list_buckets, const affine *__restrict__ points,
                                       const unsigned long long *__restrict__ count, unsigned ranges, unsigned *__restrict__ work,
                                       xyzz *__restrict__ buckets, uint8_t *__restrict__ flags, uint32_t *__restrict__ head_bucket,
                                       xyzz *__restrict__ head_point);

// ---------------------------------------------------------------------------
// 5. heads
// ---------------------------------------------------------------------------
// 32 heads per warp; one output head per warp (hb_out[w], INVALID_BUCKET if
// none).  A version with 8 heads per warp and 4-lane additions
// (msm_group4.cuh) measured slower: 0.089 -> 0.123 ms at 2^12, 0.081 ->
// 0.136 ms at 2^22 (more levels, heavier kernel).
constexpr unsigned MERGE_HEADS_PER_WARP = 32;
__global__ void merge_heads_kernel(const uint32_t *__restrict__ hb_in, const xyzz *__restrict__ hp_in, unsigned n_in, xyzz *__restrict__ buckets,
                                   uint32_t *__restrict__ hb_out, xyzz *__restrict__ hp_out);
// the same with 8 heads per warp and 4-lane additions (msm_group4.cuh), for
// levels of at most MERGE_HEADS_GROUP4_MAX heads; launched as one level of a
// chain of merge launches (enqueue_merge_heads)
constexpr unsigned MERGE_HEADS_PER_WARP_GROUP4 = 8;
__global__ void merge_heads_group4_kernel(const uint32_t *__restrict__ hb_in, const xyzz *__restrict__ hp_in, unsigned n_in,
                                          xyzz *__restrict__ buckets, uint32_t *__restrict__ hb_out, xyzz *__restrict__ hp_out);

// buckets += chunk_buckets for every slot flagged in chunk_flags
__global__ void merge_chunk_buckets_kernel(xyzz *__restrict__ buckets, uint8_t *__restrict__ flags, const xyzz *__restrict__ chunk_buckets,
                                           const uint8_t *__restrict__ chunk_flags, unsigned slots);

// ---------------------------------------------------------------------------
// 6. reduction
// ---------------------------------------------------------------------------
__global__ void reduce_groups_kernel(const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags, unsigned windows, unsigned log_b,
                                     unsigned log_m, xyzz *__restrict__ run, xyzz *__restrict__ streams);
// one level of the tree and of every live stream (see msm_kernels.cu)
__global__ void reduce_level_kernel(const xyzz *__restrict__ t_in, xyzz *__restrict__ t_out, const xyzz *__restrict__ s_in, xyzz *__restrict__ s_out,
                                    unsigned windows, unsigned log_g, unsigned level);
// the same with a group of four lanes per thread of theirs (small launches)
__global__ void reduce_groups_group4_kernel(const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags, unsigned windows, unsigned log_b,
                                            unsigned log_m, xyzz *__restrict__ run, xyzz *__restrict__ streams);
__global__ void reduce_level_group4_kernel(const xyzz *__restrict__ t_in, xyzz *__restrict__ t_out, const xyzz *__restrict__ s_in,
                                           xyzz *__restrict__ s_out, unsigned windows, unsigned log_g, unsigned level);
__global__ void gather_results_kernel(const xyzz *__restrict__ streams, const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                      unsigned windows, unsigned c, unsigned log_m, unsigned log_g, jacobian *__restrict__ results);

// stride of the per-window plain-sum streams (stream 0: G entries, stream s: G >> s)
__host__ __device__ __forceinline__ size_t stream_stride(unsigned log_g) { return (size_t)2 << log_g; }

// Stream layout per window (stride 2G): stream 0 = the G group sums "acc",
// stream s >= 1 = the G >> s odd entries of tree level s - 1.
__host__ __device__ __forceinline__ unsigned stream_offset(unsigned log_g, unsigned s) {
  const unsigned g = 1u << log_g;
  return s == 0 ? 0 : g + (g - (g >> (s - 1)));
}

__host__ __device__ __forceinline__ unsigned stream_length(unsigned log_g, unsigned s) { return s == 0 ? (1u << log_g) : (1u << log_g) >> s; }

} // namespace msm_b200
