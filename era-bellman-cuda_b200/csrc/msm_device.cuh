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
// may use digit_base[] and warp_sums[] as scratch.  AFTER() runs on every
// thread once glob[] is complete, before the tile is staged and written.
struct no_op {
  __device__ __forceinline__ void operator()() const {}
};
template <bool STABLE, bool DROP_ZEROS, class RUN_BASES, class AFTER = no_op>
__device__ __forceinline__ void scatter_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out,
                                             uint32_t *__restrict__ vals_out, size_t seg_in, size_t seg_out, unsigned base, unsigned count,
                                             unsigned shift, RUN_BASES run_bases, AFTER after = AFTER()) {
  __shared__ uint32_t s_key[SORT_TILE];
  __shared__ uint32_t s_val[SORT_TILE];
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
  after();
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    if (i < count && (!DROP_ZEROS || key[r] != ZERO_KEY)) {
      const unsigned d = sort_digit(key[r], shift);
      const unsigned pos = tile_off[d] + (STABLE ? whist[warp][d] : 0) + rank[r];
      s_key[pos] = key[r];
      s_val[pos] = val[r];
    }
  }
  __syncthreads();
#pragma unroll 4
  for (unsigned j = 0; j < SORT_ITEMS; j++) {
    const unsigned pos = j * SORT_THREADS + threadIdx.x;
    if (pos < staged) {
      const uint32_t k = s_key[pos];
      const unsigned d = sort_digit(k, shift);
      const size_t out = seg_out + glob[d] + (pos - tile_off[d]);
      keys_out[out] = k;
      vals_out[out] = s_val[pos];
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
// stable radix passes in one kernel, with decoupled look-back (the plain
// pipeline's passes after the first)
// ---------------------------------------------------------------------------
// Per (window, tile): a flag word -- LOOKBACK_NONE, LOOKBACK_AGGREGATE (the
// tile's own digit counts are in agg[tile][0..255]) or LOOKBACK_INCLUSIVE (the
// counts over this and every earlier tile of the window are in
// incl[tile][0..255]).  The counts are written first and made visible
// (__threadfence) before the flag is set; readers load the flag with acquire
// semantics before the counts.
constexpr uint32_t LOOKBACK_NONE = 0, LOOKBACK_AGGREGATE = 1, LOOKBACK_INCLUSIVE = 2;
// Polls of a batch of predecessors, one of which has published nothing yet,
// before a wait gives up (well under a second with the back-off below).  A
// predecessor took its tile earlier from the same counter, so it is resident
// and publishes its counts right after ranking: in correct operation the wait
// ends within microseconds; the limit only keeps a failure from hanging the
// GPU.
constexpr unsigned LOOKBACK_MAX_POLLS = 1u << 20;
constexpr int LOOKBACK_GAVE_UP = -2;
static_assert(SORT_THREADS == SORT_RADIX, "look-back: one digit per thread");

__device__ __forceinline__ uint32_t load_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t load_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_release(uint32_t *p, uint32_t v) { asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }

// Publishes this tile's digit counts src[0..255] (shared memory) under
// `flag`: the first warp writes them (eight per lane), makes its writes
// visible device-wide, then sets the flag.  Called by the first warp only.
__device__ __forceinline__ void lookback_publish(uint32_t *flags, uint32_t *counts, unsigned tile, const uint32_t *src, uint32_t flag) {
  const unsigned lane = threadIdx.x & 31;
  uint32_t *row = counts + (size_t)tile * SORT_RADIX;
#pragma unroll
  for (unsigned k = 0; k < SORT_RADIX / 32; k++)
    row[k * 32 + lane] = src[k * 32 + lane];
  __threadfence();
  __syncwarp();
  if (lane == 0)
    store_release(flags + tile, flag);
}

// One stable radix pass over one tile of a window segment, with run
// positions found by decoupled look-back over the window's earlier tiles:
// after ranking, the tile publishes its aggregate; the first warp then reads
// the flags of the 32 nearest earlier tiles at a time until it finds one with
// an inclusive count (waiting, bounded, while a tile between has published
// nothing), and every thread adds that inclusive count and the aggregates
// after it for its digit; the tile then publishes its own inclusive count.
// totals: the window's digit totals.  A wait that gives up sets *error and
// uses what it has (positions then only shrink, so every write stays inside
// the segment): the kernel always ends; the sort is wrong and *error says so.
__device__ __forceinline__ void lookback_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                              uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, size_t seg, unsigned tile,
                                              unsigned count, unsigned shift, uint32_t *flags, uint32_t *agg, uint32_t *incl,
                                              const uint32_t *__restrict__ totals, unsigned *error) {
  __shared__ uint32_t s_incl[SORT_RADIX]; // this tile's inclusive counts, published after the bases are known
  scatter_tile<true, false>(
      keys_in, vals_in, keys_out, vals_out, seg, seg, tile * SORT_TILE, count, shift,
      [&](const uint32_t *tile_cnt, uint32_t *glob, uint32_t *digit_base, uint32_t *warp_sums) {
        __shared__ int s_start;
        const unsigned d = threadIdx.x, lane = threadIdx.x & 31;
        const uint32_t own = tile_cnt[d];
        if (threadIdx.x < 32) {
          lookback_publish(flags, agg, tile, tile_cnt, LOOKBACK_AGGREGATE);
          int hi = (int)tile; // tiles [0, hi) are still to be examined
          int start = -1;     // nearest earlier tile with an inclusive count
          unsigned polls = 0;
          while (hi > 0) {
            const int j = hi - 1 - (int)lane;
            const uint32_t f = j >= 0 ? load_acquire(flags + j) : LOOKBACK_AGGREGATE;
            const unsigned inclusive = __ballot_sync(0xffffffffu, f == LOOKBACK_INCLUSIVE);
            const unsigned missing = __ballot_sync(0xffffffffu, f == LOOKBACK_NONE);
            const unsigned nearest = inclusive ? __ffs(inclusive) - 1 : 32;
            const unsigned before = nearest == 32 ? 0xffffffffu : (1u << nearest) - 1;
            if (missing & before) {
              if (++polls == LOOKBACK_MAX_POLLS) {
                if (lane == 0)
                  atomicOr(error, 1u);
                start = LOOKBACK_GAVE_UP;
                break;
              }
              __nanosleep(100);
              continue;
            }
            if (nearest < 32) {
              start = hi - 1 - (int)nearest;
              break;
            }
            hi -= 32;
          }
          if (lane == 0)
            s_start = start;
        }
        glob[d] = totals[d];
        __syncthreads();
        scan_256(glob, digit_base, warp_sums); // digit bases of this segment
        const int start = s_start;
        uint32_t prefix = start >= 0 ? load_relaxed(incl + (size_t)start * SORT_RADIX + d) : 0;
        if (start != LOOKBACK_GAVE_UP) {
          for (int j = start + 1; j < (int)tile; j++)
            prefix += load_relaxed(agg + (size_t)j * SORT_RADIX + d);
        } else { // add what the earlier tiles have published
          for (int j = 0; j < (int)tile; j++)
            if (load_relaxed(flags + j) != LOOKBACK_NONE)
              prefix += load_relaxed(agg + (size_t)j * SORT_RADIX + d);
        }
        glob[d] = digit_base[d] + prefix;
        s_incl[d] = prefix + own;
      },
      [&] { // the first warp publishes the inclusive counts; the others go on
        if (threadIdx.x < 32)
          lookback_publish(flags, incl, tile, s_incl, LOOKBACK_INCLUSIVE);
      });
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
