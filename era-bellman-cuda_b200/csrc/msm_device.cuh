// Device helpers shared by the MSM kernels of the plain pipeline
// (msm_kernels.cu) and of the batched pipeline (msm_batch.cu): 128-bit vector
// memory access, signed-digit extraction, and the tile-level pieces of the
// project's LSD radix sort.
#pragma once

#include "msm_kernels.cuh"

namespace msm_b200 {

// ---------------------------------------------------------------------------
// 128-bit vector memory helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ fe load_fe_streaming(const fe *p) {
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  const uint4 a = __ldcs(q), b = __ldcs(q + 1);
  fe r;
  r.l[0] = a.x, r.l[1] = a.y, r.l[2] = a.z, r.l[3] = a.w;
  r.l[4] = b.x, r.l[5] = b.y, r.l[6] = b.z, r.l[7] = b.w;
  return r;
}

__device__ __forceinline__ affine load_affine(const affine *p) {
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  const uint4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
  affine r;
  r.x.l[0] = a.x, r.x.l[1] = a.y, r.x.l[2] = a.z, r.x.l[3] = a.w;
  r.x.l[4] = b.x, r.x.l[5] = b.y, r.x.l[6] = b.z, r.x.l[7] = b.w;
  r.y.l[0] = c.x, r.y.l[1] = c.y, r.y.l[2] = c.z, r.y.l[3] = c.w;
  r.y.l[4] = d.x, r.y.l[5] = d.y, r.y.l[6] = d.z, r.y.l[7] = d.w;
  return r;
}

__device__ __forceinline__ xyzz load_xyzz(const xyzz *p) {
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  xyzz r;
  uint32_t *w = reinterpret_cast<uint32_t *>(&r);
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint4 v = q[i];
    w[4 * i + 0] = v.x;
    w[4 * i + 1] = v.y;
    w[4 * i + 2] = v.z;
    w[4 * i + 3] = v.w;
  }
  return r;
}

__device__ __forceinline__ void store_xyzz(xyzz *p, const xyzz &v) {
  uint4 *q = reinterpret_cast<uint4 *>(p);
  const uint32_t *w = reinterpret_cast<const uint32_t *>(&v);
#pragma unroll
  for (int i = 0; i < 8; i++)
    q[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}

__device__ __forceinline__ void store_jacobian(jacobian *p, const jacobian &v) {
  uint4 *q = reinterpret_cast<uint4 *>(p);
  const uint32_t *w = reinterpret_cast<const uint32_t *>(&v);
#pragma unroll
  for (int i = 0; i < 6; i++)
    q[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}

__device__ __forceinline__ uint32_t limb_at(const fe &s, unsigned k) {
  uint32_t r = 0;
#pragma unroll
  for (unsigned j = 0; j < 8; j++)
    r = (k == j) ? s.l[j] : r;
  return r;
}

// ---------------------------------------------------------------------------
// 1. digits
// ---------------------------------------------------------------------------
// Signed windows of one scalar; emit(w, key, negative) for each window.
// C != 0 fixes the window width at compile time (windows = ceil(254 / C)):
// the window loop unrolls and every limb index is a constant, which removes
// the run-time limb selection; C == 0 takes c and windows at run time.
template <unsigned C, class EMIT>
__device__ __forceinline__ void scalar_digits_fixed(const fe &scalar_mont, unsigned c_run, unsigned windows_run, EMIT emit) {
  const unsigned c = C ? C : c_run;
  const unsigned windows = C ? (RESULT_BITS + C - 1) / C : windows_run;
  fe s = fr::from_mont(scalar_mont); // canonical, < r
  // r - s (s == 0 gives r, which is never the smaller one)
  const fe m = fr::modulus();
  fe neg;
  neg.l[0] = bn254::cc::sub_cc(m.l[0], s.l[0]);
#pragma unroll
  for (int k = 1; k < 8; k++)
    neg.l[k] = bn254::cc::subc_cc(m.l[k], s.l[k]);
  const bool flip = fr::lt(neg, s);
  if (flip)
    s = neg;
  const uint32_t half = 1u << (c - 1);
  const uint32_t mask = (1u << c) - 1;
  uint32_t carry = 0;
#pragma unroll
  for (unsigned w = 0; w < windows; w++) {
    const unsigned bit = w * c;
    const unsigned limb = bit >> 5;
    const uint32_t lo = limb < 8 ? limb_at(s, limb) : 0;
    const uint32_t hi = limb + 1 < 8 ? limb_at(s, limb + 1) : 0;
    uint32_t raw = (__funnelshift_r(lo, hi, bit & 31) & mask) + carry;
    uint32_t negative = 0;
    if (raw > half) {
      raw = (mask + 1) - raw;
      negative = 1;
      carry = 1;
    } else {
      carry = 0;
    }
    emit(w, raw, negative ^ (flip ? 1u : 0u));
  }
}

template <class EMIT> __device__ __forceinline__ void scalar_digits(const fe &scalar_mont, unsigned c, unsigned windows, EMIT emit) {
  scalar_digits_fixed<0>(scalar_mont, c, windows, emit);
}

// a compile-time window width passed to generic lambdas
template <unsigned C> struct width_constant {
  static constexpr unsigned value = C;
};

// Sort key of a signed digit of magnitude m = |d| in [0, 2^(c-1)]: m - 1, so
// the keys of nonzero digits take c - 1 bits, and a zero digit wraps to
// ZERO_KEY, which the first sort pass drops.  A key's bucket slot within its
// window is m mod 2^(c-1): slot 0 holds m = 2^(c-1).
constexpr uint32_t ZERO_KEY = 0xffffffffu;
__host__ __device__ __forceinline__ uint32_t digit_key(uint32_t magnitude) { return magnitude - 1; }
__host__ __device__ __forceinline__ uint32_t key_slot(uint32_t key, uint32_t slot_mask) { return (key + 1) & slot_mask; }

// ---------------------------------------------------------------------------
// LSD radix sort, tile level (one 8-bit digit per pass)
// ---------------------------------------------------------------------------
constexpr unsigned SORT_WARPS = SORT_THREADS / 32;

__device__ __forceinline__ unsigned sort_digit(uint32_t key, unsigned shift) { return (key >> shift) & (SORT_RADIX - 1); }

// Tile histogram of `count` keys at seg_keys[base..]: out[d * out_stride] =
// number of keys whose current digit is d.  Per-warp shared counters (no
// cross-warp contention); the dominant zero digit of sparse scalars is
// counted with one ballot per warp.  DROP_ZEROS (the first pass): ZERO_KEY
// entries (zero digits, which add nothing to any bucket) are left out of the
// histogram and counted into *zero_count instead, so the scatter drops them.
template <bool DROP_ZEROS>
__device__ __forceinline__ void sort_histogram_tile(const uint32_t *__restrict__ seg_keys, unsigned base, unsigned count, unsigned shift,
                                                    uint32_t *__restrict__ out, size_t out_stride, uint32_t *__restrict__ zero_count) {
  __shared__ uint32_t hist[SORT_WARPS][SORT_RADIX];
  __shared__ uint32_t s_zero_keys;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned d = lane; d < SORT_RADIX; d += 32)
    hist[warp][d] = 0;
  if (DROP_ZEROS && threadIdx.x == 0)
    s_zero_keys = 0;
  __syncthreads();
  uint32_t zero_keys = 0;
#pragma unroll 4
  for (unsigned k = 0; k < SORT_ITEMS; k++) {
    const unsigned i = k * SORT_THREADS + threadIdx.x;
    bool valid = i < count;
    const uint32_t key = valid ? seg_keys[base + i] : 0;
    if (DROP_ZEROS) {
      const unsigned dropped = __ballot_sync(0xffffffffu, valid && key == ZERO_KEY);
      zero_keys += __popc(dropped);
      valid = valid && key != ZERO_KEY;
    }
    const unsigned d = valid ? sort_digit(key, shift) : 0;
    const unsigned zeros = __ballot_sync(0xffffffffu, valid && d == 0);
    if (valid && d != 0)
      atomicAdd(&hist[warp][d], 1u);
    if (lane == 0 && zeros)
      hist[warp][0] += __popc(zeros);
  }
  if (DROP_ZEROS && lane == 0 && zero_keys)
    atomicAdd(&s_zero_keys, zero_keys);
  __syncthreads();
  for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x) {
    uint32_t sum = 0;
#pragma unroll
    for (unsigned k = 0; k < SORT_WARPS; k++)
      sum += hist[k][d];
    out[d * out_stride] = sum;
  }
  if (DROP_ZEROS && threadIdx.x == 0 && s_zero_keys)
    atomicAdd(zero_count, s_zero_keys);
}

// One warp: exclusive prefix of row[0..len) in place, the row total into
// *total.  The row goes through in rounds of 32 consecutive entries, one per
// lane (coalesced: each load and store is one 128-byte line), scanned across
// the warp with shuffles and offset by the running total.  (Lane-contiguous
// chunks made every load touch 32 lines; at 2^22 the scan kernel took 57 us.)
__device__ __forceinline__ void sort_scan_row(uint32_t *r, unsigned len, uint32_t *__restrict__ total) {
  const unsigned lane = threadIdx.x & 31;
  uint32_t run = 0;
  for (unsigned base = 0; base < len; base += 32) {
    const unsigned t = base + lane;
    const uint32_t v = t < len ? r[t] : 0;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= (unsigned)off)
        incl += u;
    }
    if (t < len)
      r[t] = run + incl - v;
    run += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0)
    *total = run;
}

// Lanes of the warp holding the same digit d (0..SORT_RADIX; SORT_RADIX marks
// an invalid item, which only matches other invalid items): one ballot per
// bit of d.  Measured on a B200, the nine ballots beat __match_any_sync (the
// stable scatter of a 2^22 MSM: sort stage 1.29 -> 1.19 ms).
__device__ __forceinline__ unsigned warp_peers(unsigned d) {
  unsigned peers = 0xffffffffu;
#pragma unroll
  for (unsigned b = 0; b <= SORT_RADIX_BITS; b++) {
    const bool bit = (d >> b) & 1;
    const unsigned v = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? v : ~v;
  }
  return peers;
}

// Exclusive block-wide scan of 256 shared counters by the first 256 threads.
__device__ __forceinline__ void scan_256(const uint32_t *in, uint32_t *out, uint32_t *warp_sums) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t v = 0, incl = 0;
  if (threadIdx.x < SORT_RADIX) {
    v = in[threadIdx.x];
    incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= (unsigned)off)
        incl += u;
    }
    if (lane == 31)
      warp_sums[warp] = incl;
  }
  __syncthreads();
  if (threadIdx.x < SORT_RADIX) {
    uint32_t before = 0;
    for (unsigned k = 0; k < warp; k++)
      before += warp_sums[k];
    out[threadIdx.x] = before + incl - v;
  }
  __syncthreads();
}

// Scatter one tile: `count` items at seg_in + base, each to seg_out + (the
// global position of its digit's run for this tile) + (its rank among the
// tile's items of that digit).  DROP_ZEROS (the first pass): ZERO_KEY entries
// are not written (the histograms left them out).  Ranks among equal digits:
// STABLE (every pass after the first, which LSD order requires) ranks warp by
// warp, 32 consecutive items per round with warp_peers (ballots); the first
// pass may take any order and ranks with shared atomics.  The tile is then
// reordered in shared memory so that each digit's run is written to global
// memory with consecutive addresses.
//
// RUN_BASES fills glob[d] (d < SORT_RADIX), the position of this tile's run
// of digit d relative to seg_out, from the tile's digit counts tile_cnt[]; it
// is called by every thread of the block (it may synchronise the block) and
// may use digit_base[] and warp_sums[] as scratch.
template <bool STABLE, bool DROP_ZEROS, class RUN_BASES>
__device__ __forceinline__ void scatter_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                                             uint32_t *__restrict__ vals_out, size_t seg_in, size_t seg_out, unsigned base, unsigned count,
                                             unsigned shift, RUN_BASES run_bases) {
  __shared__ uint2 s_kv[SORT_TILE]; // the staged tile, key and value in one 8-byte word
  __shared__ uint32_t whist[STABLE ? SORT_WARPS : 1][SORT_RADIX];
  __shared__ uint32_t tile_cnt[SORT_RADIX], tile_off[SORT_RADIX], glob[SORT_RADIX], digit_base[SORT_RADIX], warp_sums[SORT_WARPS];
  __shared__ uint32_t staged;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned sub = warp * (32 * SORT_ITEMS); // this warp's items: base + sub + r*32 + lane
  if (STABLE) {
    for (unsigned d = lane; d < SORT_RADIX; d += 32)
      whist[warp][d] = 0;
  } else {
    for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
      tile_cnt[d] = 0;
  }
  __syncthreads();
  uint32_t key[SORT_ITEMS], val[SORT_ITEMS], rank[SORT_ITEMS];
  const unsigned lt_mask = (1u << lane) - 1;
  // every item's loads first, so that all of them are in flight together
  // (loads interleaved with the ranking rounds wait one round at a time: the
  // sort stage took 0.917 against 0.836 ms at 2^22), then the ranking
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    key[r] = i < count ? keys_in[seg_in + base + i] : 0;
    val[r] = i < count ? vals_in[seg_in + base + i] : 0;
  }
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    const bool in_tile = i < count;
    const bool valid = in_tile && (!DROP_ZEROS || key[r] != ZERO_KEY);
    const unsigned d = valid ? sort_digit(key[r], shift) : SORT_RADIX;
    if (STABLE) {
      const unsigned peers = warp_peers(d);
      const uint32_t before = valid ? whist[warp][d] : 0;
      __syncwarp();
      if (valid && lane == (unsigned)(__ffs(peers) - 1))
        whist[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    } else {
      rank[r] = valid ? atomicAdd(&tile_cnt[d], 1u) : 0;
    }
  }
  __syncthreads();
  if (STABLE) {
    // per digit: exclusive prefix over warps (warp order = item order)
    for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x) {
      uint32_t run = 0;
#pragma unroll
      for (unsigned k = 0; k < SORT_WARPS; k++) {
        const uint32_t t = whist[k][d];
        whist[k][d] = run;
        run += t;
      }
      tile_cnt[d] = run;
    }
    __syncthreads();
  }
  scan_256(tile_cnt, tile_off, warp_sums);
  if (threadIdx.x == SORT_RADIX - 1)
    staged = tile_off[SORT_RADIX - 1] + tile_cnt[SORT_RADIX - 1]; // items kept (dropped zero keys excluded)
  run_bases(static_cast<const uint32_t *>(tile_cnt), glob, digit_base, warp_sums);
  __syncthreads();
  // glob[d] becomes the offset from a staged position to its output
  // position (mod 2^32; the output position itself is below 2^32)
  for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
    glob[d] -= tile_off[d];
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    if (i < count && (!DROP_ZEROS || key[r] != ZERO_KEY)) {
      const unsigned d = sort_digit(key[r], shift);
      s_kv[tile_off[d] + (STABLE ? whist[warp][d] : 0) + rank[r]] = make_uint2(key[r], val[r]);
    }
  }
  __syncthreads();
#pragma unroll 4
  for (unsigned j = 0; j < SORT_ITEMS; j++) {
    const unsigned pos = j * SORT_THREADS + threadIdx.x;
    if (pos < staged) {
      const uint2 kv = s_kv[pos];
      const size_t out = seg_out + (uint32_t)(glob[sort_digit(kv.x, shift)] + pos);
      keys_out[out] = kv.x;
      vals_out[out] = kv.y;
    }
  }
}

// Scatter with run positions from a histogram + scan pass (the batched
// pipeline): seg_totals[0..255] are the segment's digit totals and
// tile_counts[d * count_stride] this tile's exclusive prefix over the
// segment's earlier tiles for digit d.
template <bool STABLE, bool DROP_ZEROS>
__device__ __forceinline__ void sort_scatter_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                  uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, size_t seg_in, size_t seg_out,
                                                  unsigned base, unsigned count, unsigned shift, const uint32_t *__restrict__ tile_counts,
                                                  size_t count_stride, const uint32_t *__restrict__ seg_totals) {
  scatter_tile<STABLE, DROP_ZEROS>(keys_in, vals_in, keys_out, vals_out, seg_in, seg_out, base, count, shift,
                                   [&](const uint32_t *, uint32_t *glob, uint32_t *digit_base, uint32_t *warp_sums) {
                                     for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
                                       glob[d] = seg_totals[d];
                                     __syncthreads();
                                     scan_256(glob, digit_base, warp_sums); // digit bases of this segment
                                     for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
                                       glob[d] = digit_base[d] + tile_counts[d * count_stride];
                                   });
}

// ---------------------------------------------------------------------------
// stable radix passes in one kernel, with decoupled look-back (the passes
// after the first, plain and batched pipelines)
// ---------------------------------------------------------------------------
// Per (segment, tile, digit) one 32-bit word: a status in the top two bits --
// none yet (0), LOOKBACK_AGGREGATE (the low 30 bits are the tile's own count
// of the digit) or LOOKBACK_INCLUSIVE (the count over this and every earlier
// tile of the segment) -- and the count below it.  A reader sees status and
// count together in one load, so publishing needs no fence, and each digit
// is looked back on its own.  The words start at zero (cleared before each
// pass); counts stay below 2^30 because a segment holds at most 2^29 + 2^5
// entries (chunks of at most 2^29 points; batch instances are smaller).
constexpr uint32_t LOOKBACK_AGGREGATE = 1u << 30, LOOKBACK_INCLUSIVE = 2u << 30, LOOKBACK_COUNT = LOOKBACK_AGGREGATE - 1;
// Polls of a predecessor's word that is still empty before a wait gives up
// (well under a second with the back-off below).  A predecessor took its tile
// earlier from the same ticket counter, so it is resident and publishes right
// after ranking: in correct operation the wait ends within microseconds; the
// limit only keeps a failure from hanging the GPU.
constexpr unsigned LOOKBACK_MAX_POLLS = 1u << 20;
// Predecessor words one look-back step loads together (independent loads, so
// a walk over a few aggregates costs one or two round trips to L2).
constexpr unsigned LOOKBACK_BATCH = 8;
static_assert(SORT_RADIX == 256, "look-back: one digit per thread of the first 256");

__device__ __forceinline__ uint32_t load_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_relaxed(uint32_t *p, uint32_t v) { asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }

// Digit d's count over the tiles before `tile` of its segment (words: the
// segment's [tiles][256] words, column d).  The tile's own count `own` is
// published first (tile 0 publishes it as inclusive at once); then earlier
// words are read LOOKBACK_BATCH at a time, newest first, adding counts until
// an inclusive one; an empty word means that tile has not ranked yet and is
// polled again (bounded).  Finally the inclusive count is published.  A wait
// that gives up sets *error and returns what it has added so far: a smaller
// prefix only moves this tile's (and its successors') positions down, so
// every write stays inside the segment, the kernel ends and *error reports
// the wrong order.
__device__ __forceinline__ uint32_t lookback_digit(uint32_t *words, unsigned tile, unsigned d, uint32_t own, unsigned *error) {
  uint32_t *mine = words + (size_t)tile * SORT_RADIX + d;
  if (tile == 0) {
    store_relaxed(mine, LOOKBACK_INCLUSIVE | own);
    return 0;
  }
  store_relaxed(mine, LOOKBACK_AGGREGATE | own);
  uint32_t prefix = 0;
  int j = (int)tile - 1; // newest tile not yet added
  unsigned polls = 0;
  bool done = false;
  while (!done) {
    uint32_t v[LOOKBACK_BATCH];
#pragma unroll
    for (unsigned k = 0; k < LOOKBACK_BATCH; k++) // before tile 0: an inclusive count of zero
      v[k] = j - (int)k >= 0 ? load_relaxed(words + (size_t)(j - (int)k) * SORT_RADIX + d) : LOOKBACK_INCLUSIVE;
    bool empty = false;
#pragma unroll
    for (unsigned k = 0; k < LOOKBACK_BATCH; k++) {
      if (!done && !empty) {
        if (v[k] < LOOKBACK_AGGREGATE) {
          empty = true;
        } else {
          prefix += v[k] & LOOKBACK_COUNT;
          done = v[k] >= LOOKBACK_INCLUSIVE;
          j--;
        }
      }
    }
    if (empty) {
      if (++polls == LOOKBACK_MAX_POLLS) {
        atomicOr(error, 1u);
        break;
      }
      __nanosleep(100);
    }
  }
  store_relaxed(mine, LOOKBACK_INCLUSIVE | (prefix + own));
  return prefix;
}

// Exclusive scans over the 256 digits of two sets of values at once (thread
// d < 256 passes a[d] and b[d]; other threads pass zeros): one block barrier.
// Every thread of the block must call; each block calls it once.
__device__ __forceinline__ uint2 scan2_256(uint32_t a, uint32_t b) {
  __shared__ uint2 warp_sums[SORT_RADIX / 32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t ia = a, ib = b;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t ua = __shfl_up_sync(0xffffffffu, ia, off), ub = __shfl_up_sync(0xffffffffu, ib, off);
    if (lane >= (unsigned)off) {
      ia += ua;
      ib += ub;
    }
  }
  if (threadIdx.x < SORT_RADIX && lane == 31)
    warp_sums[warp] = make_uint2(ia, ib);
  __syncthreads();
  uint32_t ba = 0, bb = 0;
  if (threadIdx.x < SORT_RADIX)
    for (unsigned k = 0; k < warp; k++) {
      ba += warp_sums[k].x;
      bb += warp_sums[k].y;
    }
  return make_uint2(ba + ia - a, bb + ib - b);
}

// Tiles of a later pass whose entries span at most LOOKBACK_SEGMENTS values
// of the key bits below `shift` rank with shared atomics per (value, digit)
// instead of ballots (see lookback_tile); one counter row per value, in the
// rows the ballot ranking keeps per warp.
constexpr unsigned LOOKBACK_SEGMENTS = 8;

// One radix pass after the first over one tile of `count` entries (at most
// THREADS * ITEMS) at seg + base, base = tile * THREADS * ITEMS, written to
// the same segment of the output arrays, so that the segment ends up sorted
// by the key bits up to shift + 8.  The input is sorted by the bits below
// `shift` (the earlier passes), so equal digits must keep the order of those
// bits; entries with equal keys up to shift + 8 may take any order (they
// fall into one bucket).  Ranking among equal digits:
//  * when the tile's entries span at most LOOKBACK_SEGMENTS values v of the
//    lower bits (known from its first and last entry, as the tile is sorted
//    by them; the common case for large windows, where a value's entries
//    fill many tiles), with shared atomics on a counter per (v - first value,
//    digit): the digit's run in the tile holds segment 0's entries, then
//    segment 1's, ... — what a stable pass would give, up to the order of
//    equal keys;
//  * otherwise stably, warp by warp, 32 consecutive items per round
//    (warp_peers), with a counter per (warp, digit).
// Then per digit: the prefix over the counter rows, the tile's count
// published and the count over earlier tiles found by look-back
// (lookback_digit; the first 256 threads, one digit each), the digit's run
// position = its total over smaller digits (totals: the segment's digit
// totals) + that prefix.  The tile is then reordered in shared memory so
// that each digit's run is written with consecutive addresses.  Needs
// lookback_smem_bytes<THREADS, ITEMS>() of dynamic shared memory.
template <unsigned THREADS, unsigned ITEMS>
__device__ __forceinline__ void lookback_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                              uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, size_t seg, unsigned tile,
                                              unsigned count, unsigned shift, uint32_t *words, const uint32_t *__restrict__ totals,
                                              unsigned *error) {
  constexpr unsigned TILE = THREADS * ITEMS, WARPS = THREADS / 32;
  static_assert(THREADS >= SORT_RADIX && THREADS % 32 == 0, "look-back tile: at least one thread per digit");
  static_assert(LOOKBACK_SEGMENTS <= WARPS, "segment counters share the per-warp counter rows");
  extern __shared__ uint2 lookback_shared[];
  uint2 *s_kv = lookback_shared;
  // counter rows: per warp (stable ranking) or per segment (atomic ranking)
  uint32_t(*rows)[SORT_RADIX] = reinterpret_cast<uint32_t(*)[SORT_RADIX]>(lookback_shared + TILE);
  __shared__ uint32_t tile_off[SORT_RADIX], delta[SORT_RADIX];
  __shared__ uint32_t staged;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned sub = warp * (32 * ITEMS); // this warp's items: base + sub + r*32 + lane
  const size_t base = (size_t)tile * TILE;
  for (unsigned d = lane; d < SORT_RADIX; d += 32)
    rows[warp][d] = 0;
  uint32_t key[ITEMS], val[ITEMS], rank[ITEMS];
  // every item's loads first, so that all of them are in flight together;
  // the tile's first and last key give the span of its lower bits
  const uint32_t lower_mask = (1u << shift) - 1;
  const uint32_t first_lower = keys_in[seg + base] & lower_mask, last_lower = keys_in[seg + base + count - 1] & lower_mask;
#pragma unroll
  for (unsigned r = 0; r < ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    key[r] = i < count ? keys_in[seg + base + i] : 0;
    val[r] = i < count ? vals_in[seg + base + i] : 0;
  }
  const bool segmented = last_lower - first_lower < LOOKBACK_SEGMENTS; // the same in every thread
  __syncthreads();
  // the counter row of an item: its segment (clamped, so that input that is
  // not sorted as it should be still stays inside the tile) or its warp
  auto row_of = [&](uint32_t k) { return segmented ? min((k & lower_mask) - first_lower, LOOKBACK_SEGMENTS - 1) : warp; };
  if (segmented) {
#pragma unroll
    for (unsigned r = 0; r < ITEMS; r++) {
      const unsigned i = sub + r * 32 + lane;
      rank[r] = i < count ? atomicAdd(&rows[row_of(key[r])][sort_digit(key[r], shift)], 1u) : 0;
    }
  } else {
    const unsigned lt_mask = (1u << lane) - 1;
#pragma unroll
    for (unsigned r = 0; r < ITEMS; r++) {
      const unsigned i = sub + r * 32 + lane;
      const bool valid = i < count;
      const unsigned d = valid ? sort_digit(key[r], shift) : SORT_RADIX;
      const unsigned peers = warp_peers(d);
      const uint32_t before = valid ? rows[warp][d] : 0;
      __syncwarp();
      if (valid && lane == (unsigned)(__ffs(peers) - 1))
        rows[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[r] = before + __popc(peers & lt_mask);
    }
  }
  __syncthreads();
  uint32_t own = 0, prefix = 0, total = 0;
  if (threadIdx.x < SORT_RADIX) {
    const unsigned d = threadIdx.x;
#pragma unroll
    for (unsigned k = 0; k < WARPS; k++) { // per digit: exclusive prefix over the rows (row order = item order)
      const uint32_t t = rows[k][d];
      rows[k][d] = own;
      own += t;
    }
    prefix = lookback_digit(words, tile, d, own, error);
    total = totals[d];
  }
  const uint2 ex = scan2_256(own, total); // the tile's runs; the segment's digit bases
  if (threadIdx.x < SORT_RADIX) {
    tile_off[threadIdx.x] = ex.x;
    delta[threadIdx.x] = ex.y + prefix - ex.x; // output position - staged position
    if (threadIdx.x == SORT_RADIX - 1)
      staged = ex.x + own;
  }
  __syncthreads();
#pragma unroll
  for (unsigned r = 0; r < ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    if (i < count) {
      const unsigned d = sort_digit(key[r], shift);
      s_kv[tile_off[d] + rows[row_of(key[r])][d] + rank[r]] = make_uint2(key[r], val[r]);
    }
  }
  __syncthreads();
#pragma unroll 4
  for (unsigned j = 0; j < ITEMS; j++) {
    const unsigned pos = j * THREADS + threadIdx.x;
    if (pos < staged) {
      const uint2 kv = s_kv[pos];
      const size_t out = seg + (uint32_t)(delta[sort_digit(kv.x, shift)] + pos);
      keys_out[out] = kv.x;
      vals_out[out] = kv.y;
    }
  }
}

// ---------------------------------------------------------------------------
// accumulation helpers
// ---------------------------------------------------------------------------
// 16-byte asynchronous global -> shared copies (L2 only: bases are not reused
// by the same SM), one commit group per base point.
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }


#ifndef ACC_MIN_BLOCKS
#define ACC_MIN_BLOCKS 4 // resident accumulation blocks per SM (caps registers at 128)
#endif

// Bucket accumulation over a list of segments of sorted (key, value) entries.
// The nonzero entries of all segments form one virtual list of M entries,
// split into `ranges` equal contiguous ranges.  Warps take 32 consecutive
// ranges at a time from a work counter (one range per lane, lengths equal to
// within one entry, so the lanes stay in step), which keeps every SM busy
// until the last ranges are handed out.  A lane walks its range, gathers the
// signed affine base of every entry (double-buffered through shared memory by
// cp.async), starts a new XYZZ accumulator when the bucket changes and
// otherwise does one mixed addition.  A bucket that starts inside the range is
// written directly (and flagged); a bucket continued from the previous range
// leaves a "head" partial sum for merge_heads_kernel.  SEG describes the
// segments (all methods device-side):
//   count()          segments
//   prefix(s)        nonzero entries before segment s (s <= count())
//   first(s), end(s) physical index of the first nonzero entry / one past the last
//   empty(s)         no nonzero entry
//   bucket(s, key)   global bucket slot of a key of segment s
//   base(s, val)     affine base of a value of segment s (sign bit ignored)
//   POINT_LIST       true for a list of stored points (point_list_segments):
//                    an entry's value is its own position, no sign, and
//                    marker points (infinity) are skipped
template <class SEG>
__device__ __forceinline__ void accumulate_range(const SEG &seg, const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, unsigned t,
                                                 unsigned long long total, unsigned long long active, xyzz *__restrict__ buckets,
                                                 uint8_t *__restrict__ flags, uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point,
                                                 uint4 (*s_base)[4][ACC_THREADS]) {
  const unsigned segments = seg.count();
  head_bucket[t] = INVALID_BUCKET;
  if (t >= active)
    return;
  const unsigned long long beg = total * t / active;
  const unsigned long long end = total * (t + 1) / active;
  unsigned w = 0;
  while (w + 1 < segments && seg.prefix(w + 1) <= beg)
    w++;
  // cursor: physical index, its segment, and the end of that segment
  size_t idx = seg.first(w) + (size_t)(beg - seg.prefix(w));
  unsigned cw = w;
  size_t seg_end = seg.end(w);
  auto advance = [&]() {
    idx++;
    if (idx == seg_end) {
      unsigned s = cw + 1;
      while (s < segments && seg.empty(s))
        s++;
      cw = s;
      if (s < segments) {
        seg_end = seg.end(s);
        idx = seg.first(s);
      }
    }
  };

  auto issue = [&](unsigned slot, unsigned s, uint32_t val) {
    const uint4 *src = reinterpret_cast<const uint4 *>(seg.base(s, val));
#pragma unroll
    for (int c = 0; c < 4; c++)
      cp_async_16(&s_base[slot][c][threadIdx.x], src + c);
    cp_async_commit();
  };
  // A base's y is never 0 (BN254 G1 has odd order, so no point has y = 0):
  // its negation is 2p - y.
  auto fetch = [&](unsigned slot, uint32_t val) {
    affine p;
    uint32_t *w32 = reinterpret_cast<uint32_t *>(&p);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const uint4 v = s_base[slot][c][threadIdx.x];
      w32[4 * c + 0] = v.x;
      w32[4 * c + 1] = v.y;
      w32[4 * c + 2] = v.z;
      w32[4 * c + 3] = v.w;
    }
    if constexpr (!SEG::POINT_LIST) {
      const fe ny = fq::neg_nonzero(p.y);
      const bool negative = val >> 31;
#pragma unroll
      for (int i = 0; i < 8; i++)
        p.y.l[i] = negative ? ny.l[i] : p.y.l[i];
    }
    return p;
  };
  auto value_at = [&](size_t i) -> uint32_t {
    if constexpr (SEG::POINT_LIST)
      return (uint32_t)i;
    else
      return vals[i];
  };
  // an infinity marker of a point list (x = all ones, never a field element)
  auto skipped = [&](const affine &p) -> bool {
    if constexpr (SEG::POINT_LIST)
      return p.x.l[7] == 0xffffffffu;
    else
      return false;
  };

  // entry 0 of the range
  uint32_t key = keys[idx];
  uint32_t val = value_at(idx);
  issue(0, cw, val);
  // does this range start in the middle of a bucket?
  const bool continued = idx > seg.first(w) && keys[idx - 1] == key;
  unsigned bucket = seg.bucket(w, key);
  const unsigned long long count = end - beg;
  // entry 1 is fetched before entry 0 is consumed
  uint32_t nkey = 0, nval = 0;
  unsigned nw = 0;
  if (count > 1) {
    advance();
    nkey = keys[idx];
    nval = value_at(idx);
    nw = cw;
    issue(1, nw, nval);
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  const affine p0 = fetch(0, val);
  xyzz acc = curve::from_affine(p0);
  bool acc_inf = skipped(p0); // a partial sum can cancel to infinity (p + (-p))
  bool first = true;
  for (unsigned long long k = 1; k < count; k++) {
    key = nkey;
    val = nval;
    const unsigned kw = nw;
    const unsigned slot = (unsigned)(k & 1);
    if (k + 1 < count) {
      advance();
      nkey = keys[idx];
      nval = value_at(idx);
      nw = cw;
      issue(slot ^ 1, nw, nval);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    const affine p = fetch(slot, val);
    const unsigned b = seg.bucket(kw, key);
    if (b != bucket) {
      if (acc_inf)
        acc = curve::infinity();
      if (first && continued) {
        head_bucket[t] = bucket;
        store_xyzz(head_point + t, acc);
      } else {
        store_xyzz(buckets + bucket, acc);
        flags[bucket] = 1;
      }
      first = false;
      bucket = b;
      acc = curve::from_affine(p);
      acc_inf = skipped(p);
    } else if (acc_inf) {
      acc = curve::from_affine(p);
      acc_inf = skipped(p);
    } else if (!skipped(p)) {
      acc = curve::add_affine_finite(acc, p, acc_inf);
    }
  }
  if (acc_inf)
    acc = curve::infinity();
  if (first && continued) {
    head_bucket[t] = bucket;
    store_xyzz(head_point + t, acc);
  } else {
    store_xyzz(buckets + bucket, acc);
    flags[bucket] = 1;
  }
}

// The work loop over all ranges (see accumulate_range).  Only the first
// min(M, ranges) ranges hold entries, so every active range holds at least one
// entry and the heads of one bucket stay contiguous (an empty range between
// them would let two merge threads update the same bucket); every range still
// writes its head slot.  *work must be 0 at launch; blocks are whole warps.
template <class SEG>
__device__ __forceinline__ void accumulate_ranges(const SEG &seg, const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                                  unsigned ranges, unsigned *__restrict__ work, xyzz *__restrict__ buckets,
                                                  uint8_t *__restrict__ flags, uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point,
                                                  uint4 (*s_base)[4][ACC_THREADS]) {
  const unsigned long long total = seg.prefix(seg.count());
  const unsigned long long active = total < ranges ? total : ranges;
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned first = 0;
    if (lane == 0)
      first = atomicAdd(work, 32u);
    first = __shfl_sync(0xffffffffu, first, 0);
    if (first >= ranges)
      return;
    if (first + lane < ranges)
      accumulate_range(seg, keys, vals, first + lane, total, active, buckets, flags, head_bucket, head_point, s_base);
  }
}

} // namespace msm_b200
