// Point arithmetic shared by a group of four lanes, for latency-bound launches
// (the final sum, the head merge, the reduction's small levels and groups).
//
// One thread alone issues every product of an XYZZ addition (14) or doubling
// (10) one after another, so with few threads in flight an operation's time
// is its issue time.  Here lanes 4g..4g+3 hold the same operands; the
// formula's independent products run on different lanes of the group in a
// few rounds and shuffles share the results, so an operation costs a few
// dependent products.  Every lane runs the same instructions on its own
// operands (no divergence inside a group), and every lane of the warp must
// call (the shuffles take the whole warp); results are the same in all four
// lanes of a group.
#pragma once

#include "msm_kernels.cuh"

namespace msm_b200 {

__device__ __forceinline__ fe shfl_fe(const fe &v, unsigned src) {
  fe r;
#pragma unroll
  for (int k = 0; k < 8; k++)
    r.l[k] = __shfl_sync(0xffffffffu, v.l[k], src);
  return r;
}

__device__ __forceinline__ fe select_fe(bool c, const fe &a, const fe &b) {
  fe r;
#pragma unroll
  for (int k = 0; k < 8; k++)
    r.l[k] = c ? a.l[k] : b.l[k];
  return r;
}

// one of four values by the lane's role in its group (register selects)
__device__ __forceinline__ fe pick4(unsigned role, const fe &a0, const fe &a1, const fe &a2, const fe &a3) {
  return select_fe(role == 0, a0, select_fe(role == 1, a1, select_fe(role == 2, a2, a3)));
}

__device__ __forceinline__ xyzz select_xyzz(bool c, const xyzz &a, const xyzz &b) {
  xyzz r;
  r.x = select_fe(c, a.x, b.x);
  r.y = select_fe(c, a.y, b.y);
  r.zz = select_fe(c, a.zz, b.zz);
  r.zzz = select_fe(c, a.zzz, b.zzz);
  return r;
}

__device__ __forceinline__ xyzz shfl_xyzz(const xyzz &v, unsigned src) {
  xyzz r;
  r.x = shfl_fe(v.x, src);
  r.y = shfl_fe(v.y, src);
  r.zz = shfl_fe(v.zz, src);
  r.zzz = shfl_fe(v.zzz, src);
  return r;
}

__device__ __forceinline__ xyzz shfl_up_xyzz(const xyzz &v, unsigned delta) {
  xyzz r;
  const uint32_t *a = reinterpret_cast<const uint32_t *>(&v);
  uint32_t *b = reinterpret_cast<uint32_t *>(&r);
#pragma unroll
  for (int i = 0; i < 32; i++)
    b[i] = __shfl_up_sync(0xffffffffu, a[i], delta);
  return r;
}

// 2 p (dbl-2008-s-1, the formula of curve::dbl) in three rounds --
// X^2 | (2Y)^2;  M^2 | X V | U V | V ZZ;  M (S - X3) - W Y | W ZZZ -- three
// dependent products instead of ten.  Infinity (ZZ = 0) maps to a point with
// ZZ = 0, i.e. to infinity.
__device__ __forceinline__ xyzz dbl_group4(const xyzz &p) {
  const unsigned lane = threadIdx.x & 31, role = lane & 3, base = lane & ~3u;
  const fe U = fq::dbl(p.y);
  const fe r1 = fq::sqr(select_fe(role == 0, p.x, U));
  const fe X2 = shfl_fe(r1, base), V = shfl_fe(r1, base + 1);
  const fe M = fq::add(fq::dbl(X2), X2);
  const fe r2 = fq::mul(pick4(role, M, p.x, U, V), pick4(role, M, V, V, p.zz));
  const fe M2 = shfl_fe(r2, base), S = shfl_fe(r2, base + 1), W = shfl_fe(r2, base + 2), ZZ3 = shfl_fe(r2, base + 3);
  xyzz r;
  r.x = fq::sub(M2, fq::dbl(S));
  const bool lead = role == 0;
  const fe r3 = fq::mul_sub_mul(select_fe(lead, M, W), select_fe(lead, fq::sub(S, r.x), p.zzz), select_fe(lead, W, fq::zero()),
                                select_fe(lead, p.y, fq::zero()));
  r.y = shfl_fe(r3, base);
  r.zzz = shfl_fe(r3, base + 1);
  r.zz = ZZ3;
  return r;
}

// p + q (add-2008-s, the formula of curve::add) in four rounds --
//   U1 = X1 ZZ2 | U2 = X2 ZZ1 | S1 = Y1 ZZZ2 | S2 = Y2 ZZZ1;
//   PP = P^2 | R^2 | ZZ1 ZZ2 | ZZZ1 ZZZ2;
//   PPP = P PP | Q = U1 PP | ZZ3 = ZZ1 ZZ2 PP;
//   Y3 = R (Q - X3) - S1 PPP | ZZZ3 = ZZZ1 ZZZ2 PPP
// -- four dependent products instead of fourteen, with the special cases of
// curve::add: an infinite operand gives the other, P = 0 gives the double of
// p (R = 0) or infinity.  The doubling is computed (by all lanes, in three
// more rounds) only when some group of the warp needs it.
__device__ __forceinline__ xyzz add_group4(const xyzz &p, const xyzz &q) {
  const unsigned lane = threadIdx.x & 31, role = lane & 3, base = lane & ~3u;
  const fe r1 = fq::mul(pick4(role, p.x, q.x, p.y, q.y), pick4(role, q.zz, p.zz, q.zzz, p.zzz));
  const fe U1 = shfl_fe(r1, base), U2 = shfl_fe(r1, base + 1), S1 = shfl_fe(r1, base + 2), S2 = shfl_fe(r1, base + 3);
  const fe P = fq::sub(U2, U1), R = fq::sub(S2, S1);
  const fe r2 = fq::mul(pick4(role, P, R, p.zz, p.zzz), pick4(role, P, R, q.zz, q.zzz));
  const fe PP = shfl_fe(r2, base), RR = shfl_fe(r2, base + 1), ZZ12 = shfl_fe(r2, base + 2), ZZZ12 = shfl_fe(r2, base + 3);
  const fe r3 = fq::mul(pick4(role, P, U1, ZZ12, ZZ12), PP);
  const fe PPP = shfl_fe(r3, base), Q = shfl_fe(r3, base + 1), ZZ3 = shfl_fe(r3, base + 2);
  xyzz r;
  r.x = fq::sub(fq::sub(RR, PPP), fq::dbl(Q));
  const bool lead = role == 0;
  const fe r4 = fq::mul_sub_mul(select_fe(lead, R, ZZZ12), select_fe(lead, fq::sub(Q, r.x), PPP), select_fe(lead, S1, fq::zero()),
                                select_fe(lead, PPP, fq::zero()));
  r.y = shfl_fe(r4, base);
  r.zzz = shfl_fe(r4, base + 1);
  r.zz = ZZ3;
  const bool p_inf = curve::is_inf(p), q_inf = curve::is_inf(q);
  const bool equal_x = !p_inf && !q_inf && fq::is_zero(P);
  const bool doubling = equal_x && fq::is_zero(R);
  if (__any_sync(0xffffffffu, doubling))
    r = select_xyzz(doubling, dbl_group4(p), r);
  if (equal_x && !doubling)
    r = curve::infinity();
  if (q_inf)
    r = p;
  if (p_inf)
    r = q;
  return r;
}

} // namespace msm_b200
