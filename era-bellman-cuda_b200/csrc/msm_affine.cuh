// Affine pairing levels: batch-affine bucket additions ahead of the XYZZ
// accumulation.
//
// After the sort, the nonzero entries of every window form bucket runs.  One
// level pairs the elements of the current list two by two -- elements 2i and
// 2i + 1 -- and, where both belong to the same bucket, replaces the pair by
// its affine sum
//     lambda = (y1 - y0) / (x1 - x0),   x = lambda^2 - x0 - x1,
//     y = lambda (x0 - x) - y0
// (a doubling takes lambda = 3 x0^2 / (2 y0)).  All the level's slope
// denominators share one field inversion by Montgomery's simultaneous
// inversion trick ("Speeding the Pollard and elliptic curve methods of
// factorization", Math. Comp. 48, 1987): per addition one product on the way
// forward and two on the way back, plus lambda, lambda^2 and y -- 5 products
// and 1 square (1,528 multiply instructions) against the 8 products and 2
// squares (2,392) of an XYZZ += affine addition.  A level roughly halves the
// list; the XYZZ accumulation (accumulate_ranges with point_list_segments)
// then adds up what is left.
//
// One level is three launches over a fixed grid of `warps` warps:
//   forward  warp g owns the pairs [P g / warps, P (g + 1) / warps) (P pairs,
//            the last one possibly a lone element), lane l the pairs
//            first + 32 k + l.  The lane walks its pairs from the last round to
//            the first, storing for each addition the product of the slope
//            denominators before it (pre) and multiplying its own in.  The
//            warp then forms, by shuffles, each lane's product of the other
//            lanes' chains and the warp's total, and counts its output
//            elements.
//   invert   one block: the inverse of every warp total (the same trick over
//            the warps, one binary-GCD inversion for the whole level) and the
//            warps' output offsets (an exclusive scan of their counts).
//   apply    the same pairs from the first round to the last, i.e. each lane's
//            chain backwards: 1/d = inv * pre, inv = inv * d, then the affine
//            sum; output positions come from ballots, so the output list keeps
//            the input order and stays sorted by bucket.
// A pair whose elements belong to different buckets passes both through; a
// sum that is infinity (P + (-P)) is written as a marker point (x = all ones,
// never a field element below p), which later levels and the XYZZ pass skip.
// Every stored coordinate is fully reduced, so equal x means equal points or
// opposite ones, and no slope denominator is ever 0 mod p.
//
// The levels are off by default (msm_b200_set_affine_levels turns them on):
// on a B200 each level's two passes over its list in memory, and the first
// level's two random gathers of every base, cost more than the multiplies
// they save (measurements with default_affine_levels in msm_host.cu).
#pragma once

#include "msm_device.cuh"

namespace msm_b200 {

constexpr uint32_t AFFINE_MARKER_WORD = 0xffffffffu; // x.l[7] of the infinity marker

__device__ __forceinline__ bool is_marker(const affine &p) { return p.x.l[7] == AFFINE_MARKER_WORD; }

__device__ __forceinline__ affine marker_point() {
  affine p;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    p.x.l[i] = AFFINE_MARKER_WORD;
    p.y.l[i] = 0;
  }
  return p;
}

__device__ __forceinline__ fe load_fe(const fe *p) {
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  const uint4 a = __ldg(q), b = __ldg(q + 1);
  fe r;
  r.l[0] = a.x, r.l[1] = a.y, r.l[2] = a.z, r.l[3] = a.w;
  r.l[4] = b.x, r.l[5] = b.y, r.l[6] = b.z, r.l[7] = b.w;
  return r;
}

__device__ __forceinline__ void store_fe(fe *p, const fe &v) {
  uint4 *q = reinterpret_cast<uint4 *>(p);
  q[0] = make_uint4(v.l[0], v.l[1], v.l[2], v.l[3]);
  q[1] = make_uint4(v.l[4], v.l[5], v.l[6], v.l[7]);
}

__device__ __forceinline__ void store_affine(affine *p, const affine &v) {
  store_fe(&p->x, v.x);
  store_fe(&p->y, v.y);
}

__device__ __forceinline__ bool fe_equal(const fe &a, const fe &b) {
  uint32_t d = 0;
#pragma unroll
  for (int i = 0; i < 8; i++)
    d |= a.l[i] ^ b.l[i];
  return d == 0;
}

__device__ __forceinline__ fe fe_select(bool c, const fe &a, const fe &b) {
  fe r;
#pragma unroll
  for (int i = 0; i < 8; i++)
    r.l[i] = c ? a.l[i] : b.l[i];
  return r;
}

template <bool UP> __device__ __forceinline__ fe shfl_fe_by(const fe &v, unsigned delta) {
  fe r;
#pragma unroll
  for (int i = 0; i < 8; i++)
    r.l[i] = UP ? __shfl_up_sync(0xffffffffu, v.l[i], delta) : __shfl_down_sync(0xffffffffu, v.l[i], delta);
  return r;
}

// For v held by every lane of the warp: *others = the product of the other
// lanes' values, *total = the product of all 32 (Kogge-Stone inclusive prefix
// and suffix products, 10 products per lane, then one more).  All lanes call.
__device__ __forceinline__ void warp_products(const fe &v, fe *others, fe *total) {
  const unsigned lane = threadIdx.x & 31;
  fe pre = v, suf = v;
#pragma unroll
  for (unsigned d = 1; d < 32; d <<= 1) {
    const fe a = fq::mul(pre, shfl_fe_by<true>(pre, d));
    const fe b = fq::mul(suf, shfl_fe_by<false>(suf, d));
    pre = fe_select(lane >= d, a, pre);
    suf = fe_select(lane + d < 32, b, suf);
  }
  const fe ep = fe_select(lane == 0, fq::one(), shfl_fe_by<true>(pre, 1));
  const fe es = fe_select(lane == 31, fq::one(), shfl_fe_by<false>(suf, 1));
  *others = fq::mul(ep, es);
  fe t;
#pragma unroll
  for (int i = 0; i < 8; i++)
    t.l[i] = __shfl_sync(0xffffffffu, pre.l[i], 31);
  *total = t;
}

// ---------------------------------------------------------------------------
// element sources
// ---------------------------------------------------------------------------
// An element of a level's input: global bucket id and a point with fully
// reduced coordinates (or the marker).
struct level_element {
  uint32_t bucket;
  affine p;
};

// Level 1: the sorted nonzero entries of the segments of SEG (the same
// virtual list that accumulate_ranges walks), each entry's signed base,
// brought to canonical form (fully reduced, y negated for a negative digit).
template <class SEG> struct segment_source {
  SEG seg;
  const uint32_t *__restrict__ keys;
  const uint32_t *__restrict__ vals;

  __device__ __forceinline__ unsigned long long count() const { return seg.prefix(seg.count()); }

  // physical index and segment of virtual element j < count()
  __device__ __forceinline__ size_t locate(unsigned long long j, unsigned &s) const {
    unsigned lo = 0, hi = seg.count(); // prefix(lo) <= j < prefix(hi)
    while (hi - lo > 1) {
      const unsigned mid = (lo + hi) >> 1;
      if (seg.prefix(mid) <= j)
        lo = mid;
      else
        hi = mid;
    }
    s = lo;
    return seg.first(lo) + (size_t)(j - seg.prefix(lo));
  }

  // bucket and x only (the forward pass)
  __device__ __forceinline__ void load_x(unsigned long long j, uint32_t &bucket, fe &x, const affine *&where, bool &negative) const {
    unsigned s;
    const size_t idx = locate(j, s);
    const uint32_t key = keys[idx], val = vals[idx];
    bucket = seg.bucket(s, key);
    where = seg.base(s, val);
    negative = val >> 31;
    x = fq::reduce_full(load_fe(&where->x));
  }

  __device__ __forceinline__ fe load_y(const affine *where, bool negative) const {
    const fe y = fq::reduce_full(load_fe(&where->y));
    return negative ? fq::reduce_full(fq::neg(y)) : y;
  }

  __device__ __forceinline__ level_element load(unsigned long long j) const {
    level_element e;
    const affine *where;
    bool negative;
    load_x(j, e.bucket, e.p.x, where, negative);
    e.p.y = load_y(where, negative);
    return e;
  }
};

// Levels 2 and later: the previous level's output list (canonical already).
struct list_source {
  const uint32_t *__restrict__ buckets;
  const affine *__restrict__ points;
  unsigned long long total;

  __device__ __forceinline__ unsigned long long count() const { return total; }

  __device__ __forceinline__ void load_x(unsigned long long j, uint32_t &bucket, fe &x, const affine *&where, bool &negative) const {
    bucket = buckets[j];
    where = points + j;
    negative = false;
    x = load_fe(&where->x);
  }

  __device__ __forceinline__ fe load_y(const affine *where, bool) const { return load_fe(&where->y); }

  __device__ __forceinline__ level_element load(unsigned long long j) const {
    level_element e;
    e.bucket = buckets[j];
    e.p = load_affine(points + j);
    return e;
  }
};

// ---------------------------------------------------------------------------
// pairs
// ---------------------------------------------------------------------------
enum pair_kind : unsigned {
  PAIR_LONE,   // element 0 alone (the list's last element): passed through
  PAIR_SPLIT,  // different buckets: both passed through
  PAIR_KEEP0,  // element 1 is the marker: element 0 passed through
  PAIR_KEEP1,  // element 0 is the marker: element 1 passed through
  PAIR_INF,    // P + (-P), or two markers: a marker
  PAIR_ADD,    // x0 != x1: affine addition
  PAIR_DOUBLE, // the same point twice: affine doubling
};

__device__ __forceinline__ unsigned pair_outputs(pair_kind k) { return k == PAIR_SPLIT ? 2u : 1u; }

// The kind of pair i of a list of m elements, and for additions and doublings
// the slope denominator d (x1 - x0, or 2 y0) and the elements.  The forward
// pass loads y only for equal x (`full` = false); the apply pass loads both
// elements whole.
template <class SRC>
__device__ __forceinline__ pair_kind classify_pair(const SRC &src, unsigned long long i, unsigned long long m, bool full, level_element &e0,
                                                   level_element &e1, fe &d) {
  const unsigned long long j = 2 * i;
  const affine *w0, *w1;
  bool n0, n1;
  if (full)
    e0 = src.load(j);
  else
    src.load_x(j, e0.bucket, e0.p.x, w0, n0);
  if (j + 1 >= m)
    return PAIR_LONE;
  if (full)
    e1 = src.load(j + 1);
  else
    src.load_x(j + 1, e1.bucket, e1.p.x, w1, n1);
  if (e0.bucket != e1.bucket)
    return PAIR_SPLIT;
  const bool m0 = is_marker(e0.p), m1 = is_marker(e1.p);
  if (m0 || m1)
    return m0 && m1 ? PAIR_INF : m0 ? PAIR_KEEP1 : PAIR_KEEP0;
  if (!fe_equal(e0.p.x, e1.p.x)) {
    d = fq::sub(e1.p.x, e0.p.x);
    return PAIR_ADD;
  }
  if (!full) {
    e0.p.y = src.load_y(w0, n0);
    e1.p.y = src.load_y(w1, n1);
  }
  // equal x: the same point (y0 == y1 != 0) or opposite points (y0 == -y1);
  // y = 0 would be a point of order 2, which BN254 G1 does not have
  if (fe_equal(e0.p.y, e1.p.y) && !fq::is_zero_exact(e0.p.y)) {
    d = fq::dbl(e0.p.y);
    return PAIR_DOUBLE;
  }
  return PAIR_INF;
}

// pairs of warp g of `warps`: [*beg, *end)
__device__ __forceinline__ void warp_pairs(unsigned long long pairs, unsigned g, unsigned warps, unsigned long long *beg, unsigned long long *end) {
  *beg = pairs * g / warps;
  *end = pairs * (g + 1) / warps;
}

template <class SRC> __device__ __forceinline__ void affine_forward(const SRC &src, const level_arrays &a, unsigned warps) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= warps)
    return; // whole warps only
  const unsigned long long m = src.count(), pairs = (m + 1) / 2;
  unsigned long long beg, end;
  warp_pairs(pairs, g, warps, &beg, &end);
  const unsigned rounds = (unsigned)((end - beg + 31) / 32);
  fe acc = fq::one();
  unsigned outputs = 0;
  for (unsigned k = rounds; k-- > 0;) {
    const unsigned long long i = beg + 32ull * k + lane;
    if (i < end) {
      level_element e0, e1;
      fe d;
      const pair_kind kind = classify_pair(src, i, m, false, e0, e1, d);
      outputs += pair_outputs(kind);
      if (kind >= PAIR_ADD) {
        store_fe(a.pre + i, acc);
        acc = fq::mul(acc, d);
      }
    }
  }
  fe others, total;
  warp_products(acc, &others, &total);
  store_fe(a.others + (size_t)g * 32 + lane, others);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    outputs += __shfl_xor_sync(0xffffffffu, outputs, o);
  if (lane == 0) {
    store_fe(a.warp_total + g, total);
    a.warp_outputs[g] = outputs;
  }
}

template <class SRC> __device__ __forceinline__ void affine_apply(const SRC &src, const level_arrays &a, unsigned warps) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= warps)
    return;
  const unsigned long long m = src.count(), pairs = (m + 1) / 2;
  unsigned long long beg, end;
  warp_pairs(pairs, g, warps, &beg, &end);
  const unsigned rounds = (unsigned)((end - beg + 31) / 32);
  // inverse of this lane's chain: 1 / (warp total) * (the other lanes' chains)
  fe inv = fq::mul(load_fe(a.warp_inverse + g), load_fe(a.others + (size_t)g * 32 + lane));
  unsigned long long out = a.warp_base[g];
  const unsigned below = (1u << lane) - 1;
  for (unsigned k = 0; k < rounds; k++) {
    const unsigned long long i = beg + 32ull * k + lane;
    const bool valid = i < end;
    level_element e0, e1;
    fe d;
    pair_kind kind = PAIR_LONE;
    if (valid)
      kind = classify_pair(src, i, m, true, e0, e1, d);
    const unsigned n = valid ? pair_outputs(kind) : 0;
    const unsigned b1 = __ballot_sync(0xffffffffu, n >= 1), b2 = __ballot_sync(0xffffffffu, n == 2);
    const unsigned long long pos = out + __popc(b1 & below) + __popc(b2 & below);
    out += __popc(b1) + __popc(b2);
    if (!valid)
      continue;
    affine r;
    switch (kind) {
    case PAIR_ADD:
    case PAIR_DOUBLE: {
      const fe dinv = fq::mul(inv, load_fe(a.pre + i));
      inv = fq::mul(inv, d);
      fe num;
      if (kind == PAIR_ADD) {
        num = fq::sub(e1.p.y, e0.p.y);
      } else {
        const fe x2 = fq::sqr(e0.p.x);
        num = fq::add(fq::dbl(x2), x2);
      }
      const fe lambda = fq::mul(num, dinv);
      const fe x = fq::sub(fq::sub(fq::sqr(lambda), e0.p.x), e1.p.x);
      const fe y = fq::sub(fq::mul(lambda, fq::sub(e0.p.x, x)), e0.p.y);
      r.x = fq::reduce_full(x);
      r.y = fq::reduce_full(y);
      break;
    }
    case PAIR_SPLIT:
      a.out_buckets[pos + 1] = e1.bucket;
      store_affine(a.out_points + pos + 1, e1.p);
      r = e0.p;
      break;
    case PAIR_KEEP1:
      r = e1.p;
      break;
    case PAIR_INF:
      r = marker_point();
      break;
    default: // PAIR_LONE, PAIR_KEEP0
      r = e0.p;
      break;
    }
    a.out_buckets[pos] = e0.bucket;
    store_affine(a.out_points + pos, r);
  }
}

// The XYZZ pass over a level's output list: one segment, bucket ids stored as
// keys, the element's own position as its value (no sign), markers skipped.
struct point_list_segments {
  static constexpr bool POINT_LIST = true;
  const affine *__restrict__ points;
  unsigned long long total;
  __device__ __forceinline__ unsigned count() const { return 1; }
  __device__ __forceinline__ unsigned long long prefix(unsigned s) const { return s ? total : 0; }
  __device__ __forceinline__ size_t first(unsigned) const { return 0; }
  __device__ __forceinline__ size_t end(unsigned) const { return (size_t)total; }
  __device__ __forceinline__ bool empty(unsigned) const { return total == 0; }
  __device__ __forceinline__ unsigned bucket(unsigned, uint32_t key) const { return key; }
  __device__ __forceinline__ const affine *base(unsigned, uint32_t val) const { return points + val; }
};

} // namespace msm_b200
