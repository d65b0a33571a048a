// Device kernels of the Pippenger MSM pipeline; see msm_kernels.cuh for the
// overall data flow.
#include "msm_affine.cuh"
#include "msm_group4.cuh"

namespace msm_b200 {

__global__ void __launch_bounds__(256) digits_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows,
                                                     uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  scalar_digits(load_fe_streaming(scalars + i), c, windows, [&](unsigned w, uint32_t magnitude, uint32_t negative) {
    const size_t out = w * window_stride(n) + i;
    keys[out] = digit_key(magnitude);
    vals[out] = i | (negative << 31);
  });
}

// The same, one block per sort tile (SORT_TILE scalars), also counting the
// tile's nonzero keys per window and radix digit for every sort pass
// (dynamic shared memory: passes x windows x 256 counters, then windows zero
// counters).  Pass 0's counts go to hist[(w * 256 + d) * tiles + tile], which
// sort_scan_kernel turns into the first radix pass's tile offsets and digit
// totals; later passes need only their digit totals, which the block adds to
// totals[(p * windows + w) * 256 + d] (zero at launch).  Each window's zero
// digits are added to zeros[w].
__global__ void __launch_bounds__(SORT_THREADS) digits_histogram_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows,
                                                                        unsigned passes, unsigned tiles, uint32_t *__restrict__ keys,
                                                                        uint32_t *__restrict__ vals, uint32_t *__restrict__ hist,
                                                                        uint32_t *__restrict__ totals, uint32_t *__restrict__ zeros) {
  extern __shared__ uint32_t s_hist[]; // [passes][windows][SORT_RADIX], then [windows] zero digits
  const unsigned counters = passes * windows * SORT_RADIX;
  uint32_t *zero_digits = s_hist + counters;
  const unsigned tile = blockIdx.x;
  for (unsigned k = threadIdx.x; k < counters + windows; k += blockDim.x)
    s_hist[k] = 0;
  __syncthreads();
  const size_t stride = window_stride(n);
  const unsigned pass_stride = windows * SORT_RADIX;
  auto tile_digits = [&](auto width) {
    constexpr unsigned C = decltype(width)::value;
    // the next scalar is loaded before this one is decomposed, so that its
    // load overlaps the decomposition, the stores and the counting
    const unsigned first = tile * SORT_TILE + threadIdx.x;
    fe next = fr::zero();
    if (first < n)
      next = load_fe_streaming(scalars + first);
    for (unsigned k = 0; k < SORT_ITEMS; k++) {
      const unsigned i = first + k * SORT_THREADS;
      const fe scalar = next;
      if (k + 1 < SORT_ITEMS && i + SORT_THREADS < n)
        next = load_fe_streaming(scalars + i + SORT_THREADS);
      if (i < n)
        scalar_digits_fixed<C>(scalar, c, windows, [&](unsigned w, uint32_t magnitude, uint32_t negative) {
          const size_t out = w * stride + i;
          const uint32_t key = digit_key(magnitude);
          keys[out] = key;
          vals[out] = i | (negative << 31);
          if (!magnitude) {
            atomicAdd(&zero_digits[w], 1u);
            return;
          }
          uint32_t *h = s_hist + w * SORT_RADIX;
          for (unsigned p = 0; p < passes; p++, h += pass_stride)
            atomicAdd(&h[(key >> (p * SORT_RADIX_BITS)) & (SORT_RADIX - 1)], 1u);
        });
    }
  };
  // the widths the size tables pick from 2^15 points on get unrolled code
  switch (c) {
  case 13: tile_digits(width_constant<13>{}); break;
  case 15: tile_digits(width_constant<15>{}); break;
  case 16: tile_digits(width_constant<16>{}); break;
  case 17: tile_digits(width_constant<17>{}); break;
  default: tile_digits(width_constant<0>{}); break;
  }
  __syncthreads();
  for (unsigned k = threadIdx.x; k < pass_stride; k += blockDim.x)
    hist[(size_t)k * tiles + tile] = s_hist[k]; // k = w * 256 + d
  for (unsigned k = pass_stride + threadIdx.x; k < counters; k += blockDim.x)
    if (s_hist[k])
      atomicAdd(&totals[k], s_hist[k]); // k = (p * windows + w) * 256 + d
  for (unsigned w = threadIdx.x; w < windows; w += blockDim.x)
    if (zero_digits[w])
      atomicAdd(&zeros[w], zero_digits[w]);
}

// Stable radix pass (8 bits at `shift`) of every window segment's nonzero
// entries [w S + zeros[w], w S + n) in one kernel, positions by decoupled
// look-back (lookback_tile).  Blocks take their tiles in launch order from
// *tile_ctr (0 at launch), so every tile a block waits for belongs to a block
// that is already running; consecutive tickets go to different windows
// (ticket = tile * windows + w), so the tiles in flight spread over all
// windows and each window's look-back stays short.  Per window: words
// [tiles][256] (look-back tiles of LOOKBACK_TILE entries), totals[256].
__global__ void __launch_bounds__(LOOKBACK_THREADS, SORT_SCATTER_MIN_BLOCKS)
    lookback_stable_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                           uint32_t *__restrict__ vals_out, unsigned n, unsigned windows, unsigned tiles, unsigned shift, uint32_t *words,
                           const uint32_t *__restrict__ totals, const uint32_t *__restrict__ zeros, unsigned *tile_ctr, unsigned *error) {
  __shared__ unsigned s_ticket;
  if (threadIdx.x == 0)
    s_ticket = atomicAdd(tile_ctr, 1u);
  __syncthreads();
  const unsigned w = s_ticket % windows, tile = s_ticket / windows;
  const unsigned skip = zeros[w], live = n - skip;
  const unsigned base = tile * LOOKBACK_TILE;
  if (base >= live) // no later tile of this window holds entries either, so none waits for this one
    return;
  lookback_tile<LOOKBACK_THREADS, LOOKBACK_ITEMS>(keys_in, vals_in, keys_out, vals_out, w * window_stride(n) + skip, tile,
                                                  min(LOOKBACK_TILE, live - base), shift, words + (size_t)w * tiles * SORT_RADIX,
                                                  totals + (size_t)w * SORT_RADIX, error);
}

// ---------------------------------------------------------------------------
// 2'. LSD radix sort with a histogram and a scan kernel per pass (window
//    counts above the digit kernel's shared-memory histograms, c <= 5),
//    one 8-bit digit per pass, independent per window segment.
//    counts layout: [window][digit][tile]; after sort_scan_kernel it holds,
//    per (window, digit), the exclusive prefix over tiles, and digit_base
//    [window][digit] the exclusive prefix over digits: an element's output
//    position is digit_base + counts + its rank among equal digits in the tile.
//    The first pass drops zero digits (they add nothing to any bucket): it
//    counts them into zeros[w] and writes the nonzero entries of window w to
//    [w S + zeros[w], w S + n), S = window_stride(n); later passes sort that
//    range only (tiles past its end have nothing to do).
// ---------------------------------------------------------------------------
template <bool FIRST>
__device__ __forceinline__ void sort_histogram_window(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles, unsigned shift,
                                                      uint32_t *__restrict__ counts, uint32_t *__restrict__ zeros) {
  const unsigned tile = blockIdx.x, w = blockIdx.y;
  const unsigned skip = FIRST ? 0 : zeros[w], live = n - skip;
  const unsigned base = tile * SORT_TILE;
  sort_histogram_tile<FIRST>(keys + w * window_stride(n) + skip, base, base < live ? min(SORT_TILE, live - base) : 0, shift,
                             counts + (size_t)w * SORT_RADIX * tiles + tile, tiles, zeros + w);
}

__global__ void __launch_bounds__(SORT_THREADS) sort_histogram_first_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles,
                                                                            unsigned shift, uint32_t *__restrict__ counts,
                                                                            uint32_t *__restrict__ zeros) {
  sort_histogram_window<true>(keys, n, tiles, shift, counts, zeros);
}

__global__ void __launch_bounds__(SORT_THREADS) sort_histogram_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles, unsigned shift,
                                                                      uint32_t *__restrict__ counts, const uint32_t *__restrict__ zeros) {
  sort_histogram_window<false>(keys, n, tiles, shift, counts, const_cast<uint32_t *>(zeros));
}

// One warp per (window, digit) row of counts (see sort_scan_row).
__global__ void __launch_bounds__(256) sort_scan_kernel(uint32_t *counts, unsigned tiles, unsigned rows, uint32_t *__restrict__ totals) {
  const unsigned row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= rows)
    return;
  sort_scan_row(counts + (size_t)row * tiles, tiles, totals + row);
}

__global__ void __launch_bounds__(SORT_THREADS, SORT_SCATTER_MIN_BLOCKS) sort_scatter_first_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                                          uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
                                                                          unsigned n, unsigned tiles, unsigned shift,
                                                                          const uint32_t *__restrict__ counts, const uint32_t *__restrict__ totals,
                                                                          const uint32_t *__restrict__ zeros) {
  const unsigned tile = blockIdx.x, w = blockIdx.y;
  const unsigned base = tile * SORT_TILE;
  const size_t seg = w * window_stride(n);
  sort_scatter_tile<false, true>(keys_in, vals_in, keys_out, vals_out, seg, seg + zeros[w], base, min(SORT_TILE, n - base), shift,
                                 counts + (size_t)w * SORT_RADIX * tiles + tile, tiles, totals + (size_t)w * SORT_RADIX);
}

__global__ void __launch_bounds__(SORT_THREADS, SORT_SCATTER_MIN_BLOCKS) sort_scatter_stable_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                                           uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
                                                                           unsigned n, unsigned tiles, unsigned shift,
                                                                           const uint32_t *__restrict__ counts, const uint32_t *__restrict__ totals,
                                                                           const uint32_t *__restrict__ zeros) {
  const unsigned tile = blockIdx.x, w = blockIdx.y;
  const unsigned skip = zeros[w], live = n - skip;
  const unsigned base = tile * SORT_TILE;
  if (base >= live)
    return;
  const size_t seg = w * window_stride(n) + skip;
  sort_scatter_tile<true, false>(keys_in, vals_in, keys_out, vals_out, seg, seg, base, min(SORT_TILE, live - base), shift,
                                 counts + (size_t)w * SORT_RADIX * tiles + tile, tiles, totals + (size_t)w * SORT_RADIX);
}

// ---------------------------------------------------------------------------
// 4. accumulation
// ---------------------------------------------------------------------------
constexpr unsigned MAX_WINDOWS = 128;

// The plain pipeline's segments: window w holds entries [w S, w S + n)
// (S = window_stride(n)), its nonzero entries last; bucket slot of a key = (w << log_b) | key_slot(key).
struct window_segments {
  static constexpr bool POINT_LIST = false;
  const affine *__restrict__ bases;
  const unsigned long long *s_first;  // shared: first nonzero entry of window w, then one past its last
  const unsigned long long *s_prefix; // shared: nonzero entries before window w
  unsigned windows, log_b;
  __device__ __forceinline__ unsigned count() const { return windows; }
  __device__ __forceinline__ unsigned long long prefix(unsigned w) const { return s_prefix[w]; }
  __device__ __forceinline__ size_t first(unsigned w) const { return s_first[2 * w]; }
  __device__ __forceinline__ size_t end(unsigned w) const { return s_first[2 * w + 1]; }
  __device__ __forceinline__ bool empty(unsigned w) const { return s_first[2 * w] == s_first[2 * w + 1]; }
  __device__ __forceinline__ unsigned bucket(unsigned w, uint32_t key) const { return (w << log_b) | key_slot(key, (1u << log_b) - 1); }
  __device__ __forceinline__ const affine *base(unsigned, uint32_t val) const { return bases + (val & 0x7fffffffu); }
};

// s_first / s_prefix of window_segments for the n-point windows (zeros[w]
// zero digits each), filled by the block.
__device__ __forceinline__ void load_window_segments(unsigned n, unsigned windows, const uint32_t *__restrict__ zeros, unsigned long long *s_first,
                                                     unsigned long long *s_prefix) {
  const size_t stride = window_stride(n);
  for (unsigned w = threadIdx.x; w < windows; w += blockDim.x) {
    s_first[2 * w] = w * stride + zeros[w];
    s_first[2 * w + 1] = w * stride + n;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long acc = 0;
    for (unsigned w = 0; w < windows; w++) {
      s_prefix[w] = acc;
      acc += s_first[2 * w + 1] - s_first[2 * w];
    }
    s_prefix[windows] = acc;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(ACC_THREADS, ACC_MIN_BLOCKS) accumulate_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                                                 const affine *__restrict__ bases, unsigned n, unsigned windows, unsigned log_b,
                                                                 const uint32_t *__restrict__ zeros, unsigned ranges, unsigned *__restrict__ work,
                                                                 xyzz *__restrict__ buckets, uint8_t *__restrict__ flags,
                                                                 uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point) {
  __shared__ unsigned long long s_first[2 * MAX_WINDOWS];
  __shared__ unsigned long long s_prefix[MAX_WINDOWS + 1];
  __shared__ uint4 s_base[2][4][ACC_THREADS];
  load_window_segments(n, windows, zeros, s_first, s_prefix);
  const window_segments seg{bases, s_first, s_prefix, windows, log_b};
  accumulate_ranges(seg, keys, vals, ranges, work, buckets, flags, head_bucket, head_point, s_base);
}

// ---------------------------------------------------------------------------
// 4a. affine pairing levels (msm_affine.cuh)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(AFFINE_FORWARD_THREADS) affine_forward_first_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                                                                      const affine *__restrict__ bases, unsigned n, unsigned windows,
                                                                                      unsigned log_b, const uint32_t *__restrict__ zeros,
                                                                                      level_arrays a, unsigned warps) {
  __shared__ unsigned long long s_first[2 * MAX_WINDOWS];
  __shared__ unsigned long long s_prefix[MAX_WINDOWS + 1];
  load_window_segments(n, windows, zeros, s_first, s_prefix);
  const segment_source<window_segments> src{window_segments{bases, s_first, s_prefix, windows, log_b}, keys, vals};
  affine_forward(src, a, warps);
}

__global__ void __launch_bounds__(AFFINE_APPLY_THREADS, AFFINE_APPLY_MIN_BLOCKS) affine_apply_first_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, const affine *__restrict__ bases, unsigned n, unsigned windows,
    unsigned log_b, const uint32_t *__restrict__ zeros, level_arrays a, unsigned warps) {
  __shared__ unsigned long long s_first[2 * MAX_WINDOWS];
  __shared__ unsigned long long s_prefix[MAX_WINDOWS + 1];
  load_window_segments(n, windows, zeros, s_first, s_prefix);
  const segment_source<window_segments> src{window_segments{bases, s_first, s_prefix, windows, log_b}, keys, vals};
  affine_apply(src, a, warps);
}

__global__ void __launch_bounds__(AFFINE_FORWARD_THREADS) affine_forward_list_kernel(const uint32_t *__restrict__ list_buckets,
                                                                                     const affine *__restrict__ points,
                                                                                     const unsigned long long *__restrict__ count, level_arrays a,
                                                                                     unsigned warps) {
  const list_source src{list_buckets, points, *count};
  affine_forward(src, a, warps);
}

__global__ void __launch_bounds__(AFFINE_APPLY_THREADS, AFFINE_APPLY_MIN_BLOCKS) affine_apply_list_kernel(const uint32_t *__restrict__ list_buckets,
                                                                                                          const affine *__restrict__ points,
                                                                                                          const unsigned long long *__restrict__ count,
                                                                                                          level_arrays a, unsigned warps) {
  const list_source src{list_buckets, points, *count};
  affine_apply(src, a, warps);
}

// Thread t takes warps [t E, (t + 1) E): its own product chain over their
// totals (warp_inverse holds each one's prefix meanwhile), then the block's
// products of the other threads' chains (warp_products within each warp, then
// across the warps), one inversion of the block total by the binary extended
// Euclidean algorithm, and the chain backwards.  The output counts are scanned
// in the same arrangement.
__global__ void __launch_bounds__(AFFINE_INVERT_THREADS) affine_invert_kernel(const fe *__restrict__ warp_total, const uint32_t *__restrict__ warp_outputs,
                                                                              unsigned warps, fe *__restrict__ warp_inverse,
                                                                              unsigned long long *__restrict__ warp_base,
                                                                              unsigned long long *__restrict__ count_out) {
  constexpr unsigned WARPS = AFFINE_INVERT_THREADS / 32;
  __shared__ fe s_total[WARPS], s_others[WARPS];
  __shared__ fe s_inverse;
  __shared__ unsigned long long s_sum[WARPS];
  const unsigned t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const unsigned per = (warps + AFFINE_INVERT_THREADS - 1) / AFFINE_INVERT_THREADS;
  const unsigned beg = min(warps, t * per), end = min(warps, beg + per);
  fe acc = fq::one();
  unsigned long long sum = 0;
  for (unsigned j = beg; j < end; j++) {
    store_fe(warp_inverse + j, acc);
    acc = fq::mul(acc, warp_total[j]);
    sum += warp_outputs[j];
  }
  fe others, total;
  warp_products(acc, &others, &total);
  unsigned long long incl = sum; // inclusive scan of the counts within the warp
#pragma unroll
  for (unsigned d = 1; d < 32; d <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d)
      incl += v;
  }
  if (lane == 31) {
    s_total[wid] = total;
    s_sum[wid] = incl;
  }
  __syncthreads();
  if (wid == 0) {
    fe o, all;
    warp_products(lane < WARPS ? s_total[lane] : fq::one(), &o, &all);
    const unsigned long long c = lane < WARPS ? s_sum[lane] : 0;
    unsigned long long ci = c;
#pragma unroll
    for (unsigned d = 1; d < 32; d <<= 1) {
      const unsigned long long v = __shfl_up_sync(0xffffffffu, ci, d);
      if (lane >= d)
        ci += v;
    }
    if (lane < WARPS) {
      s_others[lane] = o;
      s_sum[lane] = ci - c;
    }
    if (lane == WARPS - 1)
      *count_out = ci;
    if (lane == 0)
      s_inverse = fq::to_mont(fq::inverse_binary(fq::from_mont(all)));
  }
  __syncthreads();
  fe inv = fq::mul(fq::mul(s_inverse, s_others[wid]), others);
  for (unsigned j = end; j-- > beg;) {
    const fe pre = warp_inverse[j];
    warp_inverse[j] = fq::mul(inv, pre);
    inv = fq::mul(inv, warp_total[j]);
  }
  unsigned long long base = s_sum[wid] + incl - sum;
  for (unsigned j = beg; j < end; j++) {
    warp_base[j] = base;
    base += warp_outputs[j];
  }
}

__global__ void __launch_bounds__(ACC_THREADS, ACC_MIN_BLOCKS) accumulate_list_kernel(const uint32_t *__restrict__ list_buckets,
                                                                                      const affine *__restrict__ points,
                                                                                      const unsigned long long *__restrict__ count, unsigned ranges,
                                                                                      unsigned *__restrict__ work, xyzz *__restrict__ buckets,
                                                                                      uint8_t *__restrict__ flags, uint32_t *__restrict__ head_bucket,
                                                                                      xyzz *__restrict__ head_point) {
  __shared__ uint4 s_base[2][4][ACC_THREADS];
  const point_list_segments seg{points, *count};
  accumulate_ranges(seg, list_buckets, nullptr, ranges, work, buckets, flags, head_bucket, head_point, s_base);
}

// ---------------------------------------------------------------------------
// 5. fold head partial sums into their buckets
// ---------------------------------------------------------------------------
// Warp w takes heads [32 w, 32 w + 32): a segmented inclusive scan over the
// lanes (Kogge-Stone, five shuffle steps; the heads of one bucket are
// contiguous, so equal buckets at distance d mean one segment in between)
// leaves each segment's sum in its last lane.  A segment whose bucket also
// holds the head before the warp's first is a continuation and becomes the
// warp's output head; every other segment holds its bucket's first heads of
// this level and is added into the bucket (no other warp of the launch
// touches that bucket).  All lanes take every shuffle before any diverges.
__global__ void __launch_bounds__(ACC_THREADS) merge_heads_kernel(const uint32_t *__restrict__ hb_in, const xyzz *__restrict__ hp_in,
                                                                  unsigned n_in, xyzz *__restrict__ buckets, uint32_t *__restrict__ hb_out,
                                                                  xyzz *__restrict__ hp_out) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if ((unsigned long long)w * 32 >= n_in)
    return; // whole warps only
  const unsigned long long k = (unsigned long long)w * 32 + lane;
  const uint32_t b = k < n_in ? hb_in[k] : INVALID_BUCKET;
  xyzz acc = b != INVALID_BUCKET ? load_xyzz(hp_in + k) : curve::infinity();
#pragma unroll
  for (unsigned d = 1; d < 32; d <<= 1) {
    const uint32_t bo = __shfl_up_sync(0xffffffffu, b, d);
    const xyzz o = shfl_up_xyzz(acc, d);
    if (lane >= d && bo == b && b != INVALID_BUCKET)
      acc = curve::add(o, acc);
  }
  const uint32_t prev = __shfl_up_sync(0xffffffffu, b, 1), next = __shfl_down_sync(0xffffffffu, b, 1);
  const unsigned joins = __ballot_sync(0xffffffffu, lane > 0 && prev == b); // lane continues lane - 1's segment
  const unsigned first = 31 - __clz(~joins & ((2u << lane) - 1));          // first lane of this lane's segment
  const uint32_t b0 = __shfl_sync(0xffffffffu, b, 0);
  uint32_t before = INVALID_BUCKET;
  if (lane == 0 && w > 0)
    before = hb_in[(size_t)w * 32 - 1];
  before = __shfl_sync(0xffffffffu, before, 0);
  const bool continued = b0 != INVALID_BUCKET && before == b0; // lane 0's segment began in an earlier warp
  const bool last = lane == 31 || next != b;
  if (b != INVALID_BUCKET && last) {
    if (first == 0 && continued) {
      hb_out[w] = b;
      store_xyzz(hp_out + w, acc);
    } else {
      store_xyzz(buckets + b, curve::add(load_xyzz(buckets + b), acc));
    }
  }
  if (lane == 0 && !continued)
    hb_out[w] = INVALID_BUCKET;
}

// The same merge with 8 heads per warp, one per group of four lanes whose
// XYZZ additions run in rounds of independent products (msm_group4.cuh):
// three scan steps over the groups, then the bucket additions.  For the
// small later levels, where one addition's latency is the launch's.
__global__ void __launch_bounds__(ACC_THREADS) merge_heads_group4_kernel(const uint32_t *__restrict__ hb_in, const xyzz *__restrict__ hp_in,
                                                                         unsigned n_in, xyzz *__restrict__ buckets, uint32_t *__restrict__ hb_out,
                                                                         xyzz *__restrict__ hp_out) {
  constexpr unsigned GROUPS = MERGE_HEADS_PER_WARP_GROUP4;
  const unsigned lane = threadIdx.x & 31, g = lane >> 2, role = lane & 3;
  const unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if ((unsigned long long)w * GROUPS >= n_in)
    return; // whole warps only
  const unsigned long long k = (unsigned long long)w * GROUPS + g;
  const uint32_t b = k < n_in ? hb_in[k] : INVALID_BUCKET;
  xyzz acc = b != INVALID_BUCKET ? load_xyzz(hp_in + k) : curve::infinity();
#pragma unroll
  for (unsigned d = 1; d < GROUPS; d <<= 1) {
    const uint32_t bo = __shfl_up_sync(0xffffffffu, b, 4 * d);
    const xyzz o = shfl_up_xyzz(acc, 4 * d);
    const bool take = g >= d && bo == b && b != INVALID_BUCKET;
    if (__any_sync(0xffffffffu, take))
      acc = select_xyzz(take, add_group4(o, acc), acc);
  }
  const uint32_t prev = __shfl_up_sync(0xffffffffu, b, 4), next = __shfl_down_sync(0xffffffffu, b, 4);
  const unsigned join_lanes = __ballot_sync(0xffffffffu, g > 0 && prev == b); // group g continues group g - 1's segment
  unsigned joins = 0;
#pragma unroll
  for (unsigned f = 0; f < GROUPS; f++)
    joins |= ((join_lanes >> (4 * f)) & 1u) << f;
  const unsigned first = 31 - __clz(~joins & ((2u << g) - 1)); // first group of this group's segment
  const uint32_t b0 = __shfl_sync(0xffffffffu, b, 0);
  uint32_t before = INVALID_BUCKET;
  if (lane == 0 && w > 0)
    before = hb_in[(size_t)w * GROUPS - 1];
  before = __shfl_sync(0xffffffffu, before, 0);
  const bool continued = b0 != INVALID_BUCKET && before == b0; // group 0's segment began in an earlier warp
  const bool ends = b != INVALID_BUCKET && (g == GROUPS - 1 || next != b);
  const bool out_head = ends && first == 0 && continued;
  const bool into_bucket = ends && !out_head;
  const xyzz held = into_bucket ? load_xyzz(buckets + b) : curve::infinity();
  if (__any_sync(0xffffffffu, into_bucket)) {
    const xyzz sum = add_group4(held, acc);
    if (into_bucket && role == 0)
      store_xyzz(buckets + b, sum);
  }
  if (out_head && role == 0) {
    hb_out[w] = b;
    store_xyzz(hp_out + w, acc);
  }
  if (lane == 0 && !continued)
    hb_out[w] = INVALID_BUCKET;
}

// Fold the buckets of one chunk of points into the MSM's buckets (host-resident
// inputs are processed in chunks whose copies overlap the previous chunk's
// work).  One thread per bucket slot.
__global__ void __launch_bounds__(ACC_THREADS) merge_chunk_buckets_kernel(xyzz *__restrict__ buckets, uint8_t *__restrict__ flags,
                                                                          const xyzz *__restrict__ chunk_buckets,
                                                                          const uint8_t *__restrict__ chunk_flags, unsigned slots) {
  const unsigned b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= slots || !chunk_flags[b])
    return;
  const xyzz q = load_xyzz(chunk_buckets + b);
  store_xyzz(buckets + b, flags[b] ? curve::add(load_xyzz(buckets + b), q) : q);
  flags[b] = 1;
}

// ---------------------------------------------------------------------------
// 6. reduction
// ---------------------------------------------------------------------------
// Thread (w, g): slots k = g*m + i of window w, weights k (slot 0 of a window
// holds |d| = B and is excluded here).  For i = m-1 .. 1: run += X, acc += run,
// giving acc = sum_i i * X_{gm+i} and run = sum_i X_{gm+i}; then
// S_w = sum_g acc_g + m * sum_g g * run_g.
__global__ void __launch_bounds__(ACC_THREADS, REDUCE_GROUPS_MIN_BLOCKS) reduce_groups_kernel(const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                                                    unsigned windows, unsigned log_b, unsigned log_m, xyzz *__restrict__ run_out,
                                                                    xyzz *__restrict__ streams) {
  const unsigned log_g = log_b - log_m;
  const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (windows << log_g))
    return;
  const unsigned w = gid >> log_g, g = gid & ((1u << log_g) - 1);
  const unsigned base = (w << log_b) + (g << log_m);
  xyzz run = curve::infinity(), acc = curve::infinity();
  for (unsigned i = (1u << log_m) - 1; i >= 1; i--) {
    if (flags[base + i])
      run = curve::add(run, load_xyzz(buckets + base + i));
    acc = curve::add(acc, run);
  }
  if (g > 0 && flags[base])
    run = curve::add(run, load_xyzz(buckets + base));
  store_xyzz(run_out + gid, run);
  store_xyzz(streams + (size_t)w * stream_stride(log_g) + stream_offset(log_g, 0) + g, acc);
}

// Level `level` of the reduction tail (log_g launches per reduction).  Per
// window, T_level holds G >> level pair sums of the group totals run_g
// (T_0 = run_g), and every stream s <= level holds G >> level partial sums:
//   * the tree step writes the odd entries of T_level raw as the new stream
//     level + 1 (the run_g with bit `level` of g set, summed in pairs so far)
//     and the pair sums as T_level+1;
//   * every older stream takes one pairwise step, G >> level -> G >> (level+1).
// All streams therefore shrink together and hold one sum each after the last
// level.  Streams and tree are ping-ponged between levels (in = level & 1).
__global__ void __launch_bounds__(ACC_THREADS, REDUCE_LEVEL_MIN_BLOCKS) reduce_level_kernel(const xyzz *__restrict__ t_in, xyzz *__restrict__ t_out,
                                                                   const xyzz *__restrict__ s_in, xyzz *__restrict__ s_out, unsigned windows,
                                                                   unsigned log_g, unsigned level) {
  const unsigned half = (1u << log_g) >> (level + 1);
  const unsigned jobs = level + 2; // streams 0..level, then the tree
  const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= windows * jobs * half)
    return;
  const unsigned w = gid / (jobs * half), r = gid % (jobs * half);
  const unsigned job = r / half, i = r % half;
  const size_t g = (size_t)1 << log_g;
  const size_t sbase = (size_t)w * stream_stride(log_g);
  if (job <= level) {
    const size_t o = sbase + stream_offset(log_g, job);
    store_xyzz(s_out + o + i, curve::add(load_xyzz(s_in + o + 2 * i), load_xyzz(s_in + o + 2 * i + 1)));
  } else {
    const xyzz a = load_xyzz(t_in + w * g + 2 * i);
    const xyzz b = load_xyzz(t_in + w * g + 2 * i + 1);
    store_xyzz(s_out + sbase + stream_offset(log_g, level + 1) + i, b);
    if (level + 1 < log_g)
      store_xyzz(t_out + w * g + i, curve::add(a, b));
  }
}

// reduce_groups_kernel and reduce_level_kernel with one group of four lanes
// per thread of theirs (msm_group4.cuh), for launches too small to fill the
// GPU, where each addition's issue time is the launch's latency.  Groups past
// the end redo the first job and write nothing; whole warps past the end
// leave.
__global__ void __launch_bounds__(ACC_THREADS) reduce_groups_group4_kernel(const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                                                           unsigned windows, unsigned log_b, unsigned log_m,
                                                                           xyzz *__restrict__ run_out, xyzz *__restrict__ streams) {
  const unsigned log_g = log_b - log_m;
  const unsigned total = windows << log_g;
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x, role = threadIdx.x & 3;
  if ((t & ~31u) / 4 >= total)
    return;
  const bool active = t / 4 < total;
  const unsigned gid = active ? t / 4 : 0;
  const unsigned w = gid >> log_g, g = gid & ((1u << log_g) - 1);
  const unsigned base = (w << log_b) + (g << log_m);
  xyzz run = curve::infinity(), acc = curve::infinity();
  for (unsigned i = (1u << log_m) - 1; i >= 1; i--) {
    const xyzz x = flags[base + i] ? load_xyzz(buckets + base + i) : curve::infinity();
    run = add_group4(run, x);
    acc = add_group4(acc, run);
  }
  const xyzz x0 = g > 0 && flags[base] ? load_xyzz(buckets + base) : curve::infinity();
  run = add_group4(run, x0);
  if (active && role == 0) {
    store_xyzz(run_out + gid, run);
    store_xyzz(streams + (size_t)w * stream_stride(log_g) + stream_offset(log_g, 0) + g, acc);
  }
}

__global__ void __launch_bounds__(ACC_THREADS) reduce_level_group4_kernel(const xyzz *__restrict__ t_in, xyzz *__restrict__ t_out,
                                                                          const xyzz *__restrict__ s_in, xyzz *__restrict__ s_out, unsigned windows,
                                                                          unsigned log_g, unsigned level) {
  const unsigned half = (1u << log_g) >> (level + 1);
  const unsigned jobs = level + 2; // streams 0..level, then the tree
  const unsigned total = windows * jobs * half;
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x, role = threadIdx.x & 3;
  if ((t & ~31u) / 4 >= total)
    return;
  const bool active = t / 4 < total;
  const unsigned gid = active ? t / 4 : 0;
  const unsigned w = gid / (jobs * half), r = gid % (jobs * half);
  const unsigned job = r / half, i = r % half;
  const size_t g = (size_t)1 << log_g;
  const size_t sbase = (size_t)w * stream_stride(log_g);
  xyzz a, b;
  if (job <= level) {
    const size_t o = sbase + stream_offset(log_g, job);
    a = load_xyzz(s_in + o + 2 * i);
    b = load_xyzz(s_in + o + 2 * i + 1);
  } else {
    a = load_xyzz(t_in + w * g + 2 * i);
    b = load_xyzz(t_in + w * g + 2 * i + 1);
  }
  const xyzz sum = add_group4(a, b);
  if (!active || role != 0)
    return;
  if (job <= level) {
    store_xyzz(s_out + sbase + stream_offset(log_g, job) + i, sum);
  } else {
    store_xyzz(s_out + sbase + stream_offset(log_g, level + 1) + i, b);
    if (level + 1 < log_g)
      store_xyzz(t_out + w * g + i, sum);
  }
}

// Result bit i = c*w + o:  o == 0 -> stream 0;  o == c-1 -> slot 0 (|d| = B);
// log_m <= o < c-1 -> stream o - log_m + 1;  otherwise infinity.
__global__ void gather_results_kernel(const xyzz *__restrict__ streams, const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                      unsigned windows, unsigned c, unsigned log_m, unsigned log_g, jacobian *__restrict__ results) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= RESULT_BITS)
    return;
  const unsigned w = i / c, o = i % c;
  xyzz p = curve::infinity();
  if (w < windows) {
    const size_t base = (size_t)w * stream_stride(log_g);
    if (o == 0) {
      p = load_xyzz(streams + base + stream_offset(log_g, 0));
    } else if (o == c - 1) {
      const unsigned slot0 = w << (c - 1);
      if (flags[slot0])
        p = load_xyzz(buckets + slot0);
    } else if (o >= log_m && o - log_m < log_g) {
      p = load_xyzz(streams + base + stream_offset(log_g, o - log_m + 1));
    }
  }
  store_jacobian(results + i, curve::to_jacobian(p));
}

} // namespace msm_b200
