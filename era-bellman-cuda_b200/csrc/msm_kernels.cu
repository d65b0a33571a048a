// Device kernels of the Pippenger MSM pipeline; see msm_kernels.cuh for the
// overall data flow.
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
template <class EMIT> __device__ __forceinline__ void scalar_digits(const fe *__restrict__ scalars, unsigned i, unsigned c, unsigned windows, EMIT emit) {
  fe s = fr::from_mont(load_fe_streaming(scalars + i)); // canonical, < r
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

__global__ void __launch_bounds__(256) digits_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows,
                                                     uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  scalar_digits(scalars, i, c, windows, [&](unsigned w, uint32_t key, uint32_t negative) {
    const size_t out = (size_t)w * n + i;
    keys[out] = key;
    vals[out] = i | (negative << 31);
  });
}

// The same, one block per sort tile (SORT_TILE scalars), also producing the
// first radix pass's tile histograms (low 8 bits of every window's keys), so
// that pass needs no histogram kernel.  Dynamic shared memory: windows x 256
// counters.
__global__ void __launch_bounds__(SORT_THREADS) digits_histogram_kernel(const fe *__restrict__ scalars, unsigned n, unsigned c, unsigned windows,
                                                                        unsigned tiles, uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                                                        uint32_t *__restrict__ counts) {
  extern __shared__ uint32_t hist[]; // [windows][SORT_RADIX]
  const unsigned tile = blockIdx.x;
  for (unsigned k = threadIdx.x; k < windows * SORT_RADIX; k += blockDim.x)
    hist[k] = 0;
  __syncthreads();
  for (unsigned k = 0; k < SORT_ITEMS; k++) {
    const unsigned i = tile * SORT_TILE + k * SORT_THREADS + threadIdx.x;
    if (i < n)
      scalar_digits(scalars, i, c, windows, [&](unsigned w, uint32_t key, uint32_t negative) {
        const size_t out = (size_t)w * n + i;
        keys[out] = key;
        vals[out] = i | (negative << 31);
        atomicAdd(&hist[w * SORT_RADIX + (key & (SORT_RADIX - 1))], 1u);
      });
  }
  __syncthreads();
  for (unsigned k = threadIdx.x; k < windows * SORT_RADIX; k += blockDim.x)
    counts[(size_t)k * tiles + tile] = hist[k]; // k = w * 256 + d
}

// ---------------------------------------------------------------------------
// 2. LSD radix sort, one 8-bit digit per pass, independent per window segment.
//    counts layout: [window][digit][tile]; after sort_scan_kernel it holds,
//    per (window, digit), the exclusive prefix over tiles, and digit_base
//    [window][digit] the exclusive prefix over digits: an element's output
//    position is digit_base + counts + its rank among equal digits in the tile.
// ---------------------------------------------------------------------------
constexpr unsigned SORT_WARPS = SORT_THREADS / 32;

__device__ __forceinline__ unsigned sort_digit(uint32_t key, unsigned shift) { return (key >> shift) & (SORT_RADIX - 1); }

// Tile histogram: per-warp shared counters (no cross-warp contention); the
// dominant zero digit of sparse scalars is counted with one ballot per warp.
__global__ void __launch_bounds__(SORT_THREADS) sort_histogram_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned tiles,
                                                                      unsigned shift, uint32_t *__restrict__ counts) {
  __shared__ uint32_t hist[SORT_WARPS][SORT_RADIX];
  const unsigned tile = blockIdx.x, w = blockIdx.y;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned d = lane; d < SORT_RADIX; d += 32)
    hist[warp][d] = 0;
  __syncwarp();
  const uint32_t *seg = keys + (size_t)w * n;
  const unsigned base = tile * SORT_TILE;
#pragma unroll 4
  for (unsigned k = 0; k < SORT_ITEMS; k++) {
    const unsigned idx = base + k * SORT_THREADS + threadIdx.x;
    const bool valid = idx < n;
    const unsigned d = valid ? sort_digit(seg[idx], shift) : 0;
    const unsigned zeros = __ballot_sync(0xffffffffu, valid && d == 0);
    if (valid && d != 0)
      atomicAdd(&hist[warp][d], 1u);
    if (lane == 0 && zeros)
      hist[warp][0] += __popc(zeros);
  }
  __syncthreads();
  for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x) {
    uint32_t sum = 0;
#pragma unroll
    for (unsigned k = 0; k < SORT_WARPS; k++)
      sum += hist[k][d];
    counts[((size_t)w * SORT_RADIX + d) * tiles + tile] = sum;
  }
}

// One warp per (window, digit) row of counts: exclusive prefix over tiles in
// place, the row total into totals[window][digit].  Lane l scans a contiguous
// chunk of the row; the chunk sums are scanned across the warp.
__global__ void __launch_bounds__(256) sort_scan_kernel(uint32_t *counts, unsigned tiles, unsigned rows, uint32_t *__restrict__ totals) {
  const unsigned row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31;
  if (row >= rows)
    return;
  uint32_t *r = counts + (size_t)row * tiles;
  const unsigned chunk = (tiles + 31) / 32;
  const unsigned beg = min(tiles, lane * chunk), end = min(tiles, beg + chunk);
  uint32_t local = 0;
  for (unsigned t = beg; t < end; t++)
    local += r[t];
  uint32_t incl = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= (unsigned)off)
      incl += u;
  }
  uint32_t run = incl - local;
  for (unsigned t = beg; t < end; t++) {
    const uint32_t v = r[t];
    r[t] = run;
    run += v;
  }
  if (lane == 31)
    totals[row] = incl;
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

// Scatter one tile.  Ranks among equal digits: STABLE (every pass after the
// first, which LSD order requires) ranks warp by warp, 32 consecutive items
// per round with __match_any_sync; the first pass may take any order and
// ranks with shared atomics.  The tile is then reordered in shared memory so
// that each digit's run is written to global memory with consecutive
// addresses.
template <bool STABLE>
__device__ __forceinline__ void sort_scatter_tile(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                  uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, unsigned n, unsigned tiles,
                                                  unsigned shift, const uint32_t *__restrict__ counts, const uint32_t *__restrict__ totals) {
  __shared__ uint32_t s_key[SORT_TILE];
  __shared__ uint32_t s_val[SORT_TILE];
  __shared__ uint32_t whist[STABLE ? SORT_WARPS : 1][SORT_RADIX];
  __shared__ uint32_t tile_cnt[SORT_RADIX], tile_off[SORT_RADIX], glob[SORT_RADIX], digit_base[SORT_RADIX], warp_sums[SORT_WARPS];
  const unsigned tile = blockIdx.x, w = blockIdx.y;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t seg = (size_t)w * n;
  const unsigned base = tile * SORT_TILE;
  const unsigned count = min(SORT_TILE, n - base);
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
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    const bool valid = i < count;
    key[r] = valid ? keys_in[seg + base + i] : 0;
    val[r] = valid ? vals_in[seg + base + i] : 0;
    const unsigned d = valid ? sort_digit(key[r], shift) : SORT_RADIX;
    if (STABLE) {
      const unsigned peers = __match_any_sync(0xffffffffu, d);
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
  for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
    glob[d] = totals[(size_t)w * SORT_RADIX + d];
  __syncthreads();
  scan_256(glob, digit_base, warp_sums); // digit bases of this window
  for (unsigned d = threadIdx.x; d < SORT_RADIX; d += blockDim.x)
    glob[d] = digit_base[d] + counts[((size_t)w * SORT_RADIX + d) * tiles + tile];
#pragma unroll
  for (unsigned r = 0; r < SORT_ITEMS; r++) {
    const unsigned i = sub + r * 32 + lane;
    if (i < count) {
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
    if (pos < count) {
      const uint32_t k = s_key[pos];
      const unsigned d = sort_digit(k, shift);
      const size_t out = seg + glob[d] + (pos - tile_off[d]);
      keys_out[out] = k;
      vals_out[out] = s_val[pos];
    }
  }
}

__global__ void __launch_bounds__(SORT_THREADS) sort_scatter_first_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                                          uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
                                                                          unsigned n, unsigned tiles, unsigned shift,
                                                                          const uint32_t *__restrict__ counts,
                                                                          const uint32_t *__restrict__ totals) {
  sort_scatter_tile<false>(keys_in, vals_in, keys_out, vals_out, n, tiles, shift, counts, totals);
}

__global__ void __launch_bounds__(SORT_THREADS) sort_scatter_stable_kernel(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                                                                           uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
                                                                           unsigned n, unsigned tiles, unsigned shift,
                                                                           const uint32_t *__restrict__ counts,
                                                                           const uint32_t *__restrict__ totals) {
  sort_scatter_tile<true>(keys_in, vals_in, keys_out, vals_out, n, tiles, shift, counts, totals);
}

// ---------------------------------------------------------------------------
// 3. first nonzero key of each sorted window
// ---------------------------------------------------------------------------
__global__ void zero_counts_kernel(const uint32_t *__restrict__ keys, unsigned n, unsigned windows, uint32_t *__restrict__ zeros) {
  const unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= windows)
    return;
  const uint32_t *seg = keys + (size_t)w * n;
  unsigned lo = 0, hi = n; // first index with key != 0
  while (lo < hi) {
    const unsigned mid = (lo + hi) >> 1;
    if (seg[mid] == 0)
      lo = mid + 1;
    else
      hi = mid;
  }
  zeros[w] = lo;
}

// ---------------------------------------------------------------------------
// 4. accumulation
// ---------------------------------------------------------------------------
constexpr unsigned MAX_WINDOWS = 128;
#ifndef ACC_MIN_BLOCKS
#define ACC_MIN_BLOCKS 4 // resident accumulation blocks per SM (caps registers at 128)
#endif

struct entry_cursor {
  size_t idx;       // physical index into keys / vals
  unsigned w;       // window of idx
  size_t seg_end;   // (w + 1) * n
};

__device__ __forceinline__ void cursor_advance(entry_cursor &cur, unsigned n, unsigned windows, const uint32_t *s_zeros) {
  cur.idx++;
  if (cur.idx == cur.seg_end) {
    unsigned w = cur.w + 1;
    while (w < windows && s_zeros[w] == n)
      w++;
    cur.w = w;
    cur.seg_end = (size_t)(w + 1) * n;
    cur.idx = (size_t)w * n + (w < windows ? s_zeros[w] : 0);
  }
}

// A base's y is never 0 (BN254 G1 has odd order, so no point has y = 0):
// its negation is 2p - y.
__device__ __forceinline__ affine signed_base(const affine *__restrict__ bases, uint32_t val) {
  affine p = load_affine(bases + (val & 0x7fffffffu));
  const fe ny = fq::neg_nonzero(p.y);
  const bool negative = val >> 31;
#pragma unroll
  for (int i = 0; i < 8; i++)
    p.y.l[i] = negative ? ny.l[i] : p.y.l[i];
  return p;
}

// 16-byte asynchronous global -> shared copies (L2 only: bases are not reused
// by the same SM), one commit group per base point.
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }

__global__ void __launch_bounds__(ACC_THREADS, ACC_MIN_BLOCKS) accumulate_kernel(const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
                                                                 const affine *__restrict__ bases, unsigned n, unsigned windows, unsigned log_b,
                                                                 const uint32_t *__restrict__ zeros, unsigned total_threads,
                                                                 xyzz *__restrict__ buckets, uint8_t *__restrict__ flags,
                                                                 uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point) {
  __shared__ uint32_t s_zeros[MAX_WINDOWS];
  __shared__ unsigned long long s_prefix[MAX_WINDOWS + 1];
  // two base-point slots per thread, chunk-major: [slot][16-byte chunk][thread]
  __shared__ uint4 s_base[2][4][ACC_THREADS];
  for (unsigned w = threadIdx.x; w < windows; w += blockDim.x)
    s_zeros[w] = zeros[w];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long acc = 0;
    for (unsigned w = 0; w < windows; w++) {
      s_prefix[w] = acc;
      acc += n - s_zeros[w];
    }
    s_prefix[windows] = acc;
  }
  __syncthreads();
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total_threads)
    return;
  // Only the first min(total, total_threads) ranges are used, so every active
  // range holds at least one entry and the heads of one bucket stay
  // contiguous (an empty range between them would let two merge threads
  // update the same bucket).
  const unsigned long long total = s_prefix[windows];
  const unsigned long long active = total < total_threads ? total : total_threads;
  head_bucket[t] = INVALID_BUCKET;
  if (t >= active)
    return;
  const unsigned long long beg = total * t / active;
  const unsigned long long end = total * (t + 1) / active;
  unsigned w = 0;
  while (w + 1 < windows && s_prefix[w + 1] <= beg)
    w++;
  entry_cursor cur;
  cur.w = w;
  cur.seg_end = (size_t)(w + 1) * n;
  cur.idx = (size_t)w * n + s_zeros[w] + (size_t)(beg - s_prefix[w]);
  const uint32_t slot_mask = (1u << log_b) - 1;

  auto issue = [&](unsigned slot, uint32_t val) {
    const uint4 *src = reinterpret_cast<const uint4 *>(bases + (val & 0x7fffffffu));
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
    const fe ny = fq::neg_nonzero(p.y);
    const bool negative = val >> 31;
#pragma unroll
    for (int i = 0; i < 8; i++)
      p.y.l[i] = negative ? ny.l[i] : p.y.l[i];
    return p;
  };

  // entry 0 of the range
  uint32_t key = keys[cur.idx];
  uint32_t val = vals[cur.idx];
  issue(0, val);
  // does this range start in the middle of a bucket?
  const bool continued = cur.idx > (size_t)w * n + s_zeros[w] && keys[cur.idx - 1] == key;
  unsigned bucket = (cur.w << log_b) | (key & slot_mask);
  const unsigned long long count = end - beg;
  // entry 1 is fetched before entry 0 is consumed
  uint32_t nkey = 0, nval = 0;
  unsigned nw = 0;
  if (count > 1) {
    cursor_advance(cur, n, windows, s_zeros);
    nkey = keys[cur.idx];
    nval = vals[cur.idx];
    nw = cur.w;
    issue(1, nval);
    cp_async_wait<1>();
  } else {
    cp_async_wait<0>();
  }
  xyzz acc = curve::from_affine(fetch(0, val));
  bool acc_inf = false; // a partial sum can cancel to infinity (p + (-p))
  bool first = true;
  for (unsigned long long k = 1; k < count; k++) {
    key = nkey;
    val = nval;
    const unsigned kw = nw;
    const unsigned slot = (unsigned)(k & 1);
    if (k + 1 < count) {
      cursor_advance(cur, n, windows, s_zeros);
      nkey = keys[cur.idx];
      nval = vals[cur.idx];
      nw = cur.w;
      issue(slot ^ 1, nval);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    const affine p = fetch(slot, val);
    const unsigned b = (kw << log_b) | (key & slot_mask);
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
      acc_inf = false;
    } else if (acc_inf) {
      acc = curve::from_affine(p);
      acc_inf = false;
    } else {
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

// ---------------------------------------------------------------------------
// 5. fold head partial sums into their buckets
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(ACC_THREADS) merge_heads_kernel(const uint32_t *__restrict__ hb_in, const xyzz *__restrict__ hp_in,
                                                                  unsigned n_in, unsigned chunk, xyzz *__restrict__ buckets,
                                                                  uint32_t *__restrict__ hb_out, xyzz *__restrict__ hp_out) {
  const unsigned u = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long beg = (unsigned long long)u * chunk;
  if (beg >= n_in)
    return;
  const unsigned end = (unsigned)min((unsigned long long)n_in, beg + chunk);
  hb_out[u] = INVALID_BUCKET;
  unsigned bucket = INVALID_BUCKET;
  bool head_is_continuation = false, seen = false;
  xyzz acc;
  for (unsigned k = (unsigned)beg; k < end; k++) {
    const unsigned b = hb_in[k];
    if (b == INVALID_BUCKET)
      continue;
    const xyzz p = load_xyzz(hp_in + k);
    if (b != bucket) {
      if (bucket != INVALID_BUCKET) {
        if (head_is_continuation) {
          hb_out[u] = bucket;
          store_xyzz(hp_out + u, acc);
        } else {
          store_xyzz(buckets + bucket, curve::add(load_xyzz(buckets + bucket), acc));
        }
      }
      head_is_continuation = !seen && k == beg && k > 0 && hb_in[k - 1] == b;
      seen = true;
      bucket = b;
      acc = p;
    } else {
      acc = curve::add(acc, p);
    }
  }
  if (bucket != INVALID_BUCKET) {
    if (head_is_continuation) {
      hb_out[u] = bucket;
      store_xyzz(hp_out + u, acc);
    } else {
      store_xyzz(buckets + bucket, curve::add(load_xyzz(buckets + bucket), acc));
    }
  }
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
// Stream layout per window (stride 2G): stream 0 = the G group sums "acc",
// stream s >= 1 = the G >> s odd entries of tree level s - 1.
__host__ __device__ __forceinline__ unsigned stream_offset(unsigned log_g, unsigned s) {
  const unsigned g = 1u << log_g;
  return s == 0 ? 0 : g + (g - (g >> (s - 1)));
}

__host__ __device__ __forceinline__ unsigned stream_length(unsigned log_g, unsigned s) { return s == 0 ? (1u << log_g) : (1u << log_g) >> s; }

// Thread (w, g): slots k = g*m + i of window w, weights k (slot 0 of a window
// holds |d| = B and is excluded here).  For i = m-1 .. 1: run += X, acc += run,
// giving acc = sum_i i * X_{gm+i} and run = sum_i X_{gm+i}; then
// S_w = sum_g acc_g + m * sum_g g * run_g.
__global__ void __launch_bounds__(ACC_THREADS) reduce_groups_kernel(const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
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

// Tree level `level`: T_{level} has G >> level entries per window (stride G).
// Odd entries go to stream level + 1; pair sums form T_{level+1}.
__global__ void __launch_bounds__(ACC_THREADS) reduce_tree_kernel(const xyzz *__restrict__ t_in, xyzz *__restrict__ t_out,
                                                                  xyzz *__restrict__ streams, unsigned windows, unsigned log_g,
                                                                  unsigned level) {
  const unsigned half = (1u << log_g) >> (level + 1);
  const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= windows * half)
    return;
  const unsigned w = gid / half, i = gid % half;
  const size_t g = (size_t)1 << log_g;
  const xyzz a = load_xyzz(t_in + w * g + 2 * i);
  const xyzz b = load_xyzz(t_in + w * g + 2 * i + 1);
  store_xyzz(streams + (size_t)w * stream_stride(log_g) + stream_offset(log_g, level + 1) + i, b);
  if (level + 1 < log_g)
    store_xyzz(t_out + w * g + i, curve::add(a, b));
}

// One plain-sum pass: every stream of length L (as of divisor_in) shrinks to
// ceil(L / fanin); layout unchanged.
__global__ void __launch_bounds__(ACC_THREADS) reduce_streams_kernel(const xyzz *__restrict__ in, xyzz *__restrict__ out, unsigned windows,
                                                                     unsigned log_g, unsigned fanin, unsigned divisor_in) {
  const unsigned streams_per_window = log_g + 1;
  const unsigned sid = blockIdx.y;
  const unsigned w = sid / streams_per_window, s = sid % streams_per_window;
  if (w >= windows)
    return;
  const unsigned len0 = stream_length(log_g, s);
  const unsigned len_in = (len0 + divisor_in - 1) / divisor_in;
  const unsigned len_out = (len_in + fanin - 1) / fanin;
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= len_out)
    return;
  const size_t base = (size_t)w * stream_stride(log_g) + stream_offset(log_g, s);
  xyzz acc = curve::infinity();
  for (unsigned f = 0; f < fanin; f++) {
    const unsigned k = q * fanin + f;
    if (k < len_in)
      acc = curve::add(acc, load_xyzz(in + base + k));
  }
  store_xyzz(out + base + q, acc);
}

// Result bit i = c*w + o:  o == 0 -> stream 0;  o == c-1 -> slot 0 (|d| = B);
// log_m <= o < c-1 -> stream o - log_m + 1;  otherwise infinity.
__global__ void gather_results_kernel(const xyzz *__restrict__ streams, const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                      unsigned windows, unsigned c, unsigned log_m, unsigned log_g, unsigned divisor,
                                      jacobian *__restrict__ results) {
  (void)divisor;
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
