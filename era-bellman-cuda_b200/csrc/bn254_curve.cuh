// BN254 G1 (y^2 = x^3 + 3 over Fq) point arithmetic for bucket accumulation.
//
// Coordinates are Montgomery-form Fq values kept in [0, 2p) (see
// bn254_field.cuh).  Buckets use extended Jacobian "XYZZ" coordinates
// (x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2; infinity iff ZZ == 0), the
// representation of the reference (src/ec.cuh:211-281).  Formulas are the
// published XYZZ formulas (hyperelliptic.org EFD, "g1p/auto-shortw-xyzz"):
//   madd-2008-s   XYZZ + affine          (reference src/ec.cuh:555-597)
//   add-2008-s    XYZZ + XYZZ            (reference src/ec.cuh:495-546)
//   dbl-2008-s-1  / mdbl-2008-s-1        (reference src/ec.cuh:416-487)
// with the equal-point and opposite-point cases handled explicitly.
#pragma once

#include "bn254_field.cuh"

namespace bn254 {

struct BN_ALIGN(16) affine {
  fe x, y;
};

struct BN_ALIGN(16) xyzz {
  fe x, y, zz, zzz;
};

struct BN_ALIGN(16) jacobian {
  fe x, y, z;
};

struct curve {
  static BN_HD xyzz infinity() {
    xyzz r;
    r.x = fq::zero();
    r.y = fq::one();
    r.zz = fq::zero();
    r.zzz = fq::zero();
    return r;
  }

  static BN_HD bool is_inf(const xyzz &p) { return fq::is_zero(p.zz); }

  static BN_HD xyzz from_affine(const affine &a) {
    xyzz r;
    r.x = a.x;
    r.y = a.y;
    r.zz = fq::one();
    r.zzz = fq::one();
    return r;
  }

  static BN_HD affine neg(const affine &a) {
    affine r;
    r.x = a.x;
    r.y = fq::neg(a.y);
    return r;
  }

  // 2 * a for an affine a (mdbl-2008-s-1): U = 2Y, V = U^2, W = U V,
  // S = X V, M = 3 X^2, X3 = M^2 - 2S, Y3 = M (S - X3) - W Y, ZZ3 = V, ZZZ3 = W.
  static BN_HD_COLD xyzz dbl_affine(const affine &a) {
    const fe U = fq::dbl(a.y);
    const fe V = fq::sqr(U);
    const fe W = fq::mul(U, V);
    const fe S = fq::mul(a.x, V);
    const fe X2 = fq::sqr(a.x);
    const fe M = fq::add(fq::dbl(X2), X2);
    xyzz r;
    r.x = fq::sub(fq::sqr(M), fq::dbl(S));
    r.y = fq::mul_sub_mul(M, fq::sub(S, r.x), W, a.y);
    r.zz = V;
    r.zzz = W;
    return r;
  }

  // 2 * p (dbl-2008-s-1): as above with ZZ3 = V ZZ1, ZZZ3 = W ZZZ1.
  static BN_HD_COLD xyzz dbl(const xyzz &p) {
    if (is_inf(p))
      return p;
    const fe U = fq::dbl(p.y);
    const fe V = fq::sqr(U);
    const fe W = fq::mul(U, V);
    const fe S = fq::mul(p.x, V);
    const fe X2 = fq::sqr(p.x);
    const fe M = fq::add(fq::dbl(X2), X2);
    xyzz r;
    r.x = fq::sub(fq::sqr(M), fq::dbl(S));
    r.y = fq::mul_sub_mul(M, fq::sub(S, r.x), W, p.y);
    r.zz = fq::mul(V, p.zz);
    r.zzz = fq::mul(W, p.zzz);
    return r;
  }

  // p + a (madd-2008-s):
  //   U2 = x2 ZZ1, S2 = y2 ZZZ1, P = U2 - X1, R = S2 - Y1,
  //   PP = P^2, PPP = P PP, Q = X1 PP,
  //   X3 = R^2 - PPP - 2Q, Y3 = R (Q - X3) - Y1 PPP, ZZ3 = ZZ1 PP, ZZZ3 = ZZZ1 PPP.
  // Multiplication cost: 6 mul + 2 sqr + one a*b - c*d.
  static BN_HD xyzz add_affine(const xyzz &p, const affine &a) {
    if (is_inf(p))
      return from_affine(a);
    const fe U2 = fq::mul(a.x, p.zz);
    const fe S2 = fq::mul(a.y, p.zzz);
    const fe P = fq::sub(U2, p.x);
    const fe R = fq::sub(S2, p.y);
    if (fq::is_zero(P)) {
      if (fq::is_zero(R))
        return dbl_affine(a); // p == a
      return infinity();      // p == -a
    }
    const fe PP = fq::sqr(P);
    const fe PPP = fq::mul(P, PP);
    const fe Q = fq::mul(p.x, PP);
    xyzz r;
    r.x = fq::sub(fq::sub(fq::sqr(R), PPP), fq::dbl(Q));
    r.y = fq::mul_sub_mul(R, fq::sub(Q, r.x), p.y, PPP);
    r.zz = fq::mul(p.zz, PP);
    r.zzz = fq::mul(p.zzz, PPP);
    return r;
  }

  // p + a for a finite accumulator p (no test of p's ZZ): the accumulation
  // loop tracks infinity itself.  Sets became_inf when the sum is infinity
  // (p == -a); the returned point is then unspecified.
  static BN_HD xyzz add_affine_finite(const xyzz &p, const affine &a, bool &became_inf) {
    const fe U2 = fq::mul(a.x, p.zz);
    const fe S2 = fq::mul(a.y, p.zzz);
    const fe P = fq::sub(U2, p.x);
    const fe R = fq::sub(S2, p.y);
    if (fq::is_zero(P)) {
      if (fq::is_zero(R))
        return dbl_affine(a); // p == a
      became_inf = true;      // p == -a
      return p;
    }
    const fe PP = fq::sqr(P);
    const fe PPP = fq::mul(P, PP);
    const fe Q = fq::mul(p.x, PP);
    xyzz r;
    r.x = fq::sub(fq::sub(fq::sqr(R), PPP), fq::dbl(Q));
    r.y = fq::mul_sub_mul(R, fq::sub(Q, r.x), p.y, PPP);
    r.zz = fq::mul(p.zz, PP);
    r.zzz = fq::mul(p.zzz, PPP);
    return r;
  }

  // p + q (add-2008-s):
  //   U1 = X1 ZZ2, U2 = X2 ZZ1, S1 = Y1 ZZZ2, S2 = Y2 ZZZ1, P = U2 - U1, R = S2 - S1,
  //   PP = P^2, PPP = P PP, Q = U1 PP, X3 = R^2 - PPP - 2Q,
  //   Y3 = R (Q - X3) - S1 PPP, ZZ3 = ZZ1 ZZ2 PP, ZZZ3 = ZZZ1 ZZZ2 PPP.
  static BN_HD xyzz add(const xyzz &p, const xyzz &q) {
    if (is_inf(p))
      return q;
    if (is_inf(q))
      return p;
    const fe U1 = fq::mul(p.x, q.zz);
    const fe U2 = fq::mul(q.x, p.zz);
    const fe S1 = fq::mul(p.y, q.zzz);
    const fe S2 = fq::mul(q.y, p.zzz);
    const fe P = fq::sub(U2, U1);
    const fe R = fq::sub(S2, S1);
    if (fq::is_zero(P)) {
      if (fq::is_zero(R))
        return dbl(p);
      return infinity();
    }
    const fe PP = fq::sqr(P);
    const fe PPP = fq::mul(P, PP);
    const fe Q = fq::mul(U1, PP);
    xyzz r;
    r.x = fq::sub(fq::sub(fq::sqr(R), PPP), fq::dbl(Q));
    r.y = fq::mul_sub_mul(R, fq::sub(Q, r.x), S1, PPP);
    r.zz = fq::mul(fq::mul(p.zz, q.zz), PP);
    r.zzz = fq::mul(fq::mul(p.zzz, q.zzz), PPP);
    return r;
  }

  // Jacobian (X, Y, Z; x = X/Z^2, y = Y/Z^3) -> XYZZ (X, Y, Z^2, Z^3); the
  // Jacobian infinity (Z = 0) gives ZZ = 0, the XYZZ infinity.
  static BN_HD xyzz from_jacobian(const jacobian &p) {
    xyzz r;
    r.x = p.x;
    r.y = p.y;
    r.zz = fq::sqr(p.z);
    r.zzz = fq::mul(r.zz, p.z);
    return r;
  }

  // Canonical affine output: x and y in standard (not Montgomery) form,
  // fully reduced; true, with x = y = 0, for infinity.  One binary inversion
  // of ZZ ZZZ gives 1/ZZ = ZZZ / (ZZ ZZZ) and 1/ZZZ = ZZ / (ZZ ZZZ).
  static BN_HD_COLD bool to_affine_standard(const xyzz &p, fe &x, fe &y) {
    if (is_inf(p)) {
      x = fq::zero();
      y = fq::zero();
      return true;
    }
    const fe inv = fq::to_mont(fq::inverse_binary(fq::from_mont(fq::mul(p.zz, p.zzz))));
    x = fq::from_mont(fq::mul(p.x, fq::mul(p.zzz, inv)));
    y = fq::from_mont(fq::mul(p.y, fq::mul(p.zz, inv)));
    return false;
  }

  // XYZZ -> affine for a finite p: one inversion of ZZ ZZZ gives both
  // 1/ZZ = ZZZ / (ZZ ZZZ) and 1/ZZZ = ZZ / (ZZ ZZZ).  Output fully reduced.
  static BN_HD_COLD affine to_affine(const xyzz &p) {
    const fe inv = fq::inverse(fq::mul(p.zz, p.zzz));
    affine a;
    a.x = fq::reduce_full(fq::mul(p.x, fq::mul(p.zzz, inv)));
    a.y = fq::reduce_full(fq::mul(p.y, fq::mul(p.zz, inv)));
    return a;
  }

  // XYZZ -> Jacobian (x = X/Z^2, y = Y/Z^3) with Z = ZZZ: since ZZ^3 = ZZZ^2,
  // X_J = X ZZ^2 and Y_J = Y ZZZ^2.  Output fully reduced; infinity is
  // (0, 1, 0) in Montgomery form, the reference's encoding (src/ec.cuh:139).
  static BN_HD jacobian to_jacobian(const xyzz &p) {
    jacobian r;
    if (is_inf(p)) {
      r.x = fq::zero();
      r.y = fq::one();
      r.z = fq::zero();
      return r;
    }
    r.x = fq::reduce_full(fq::mul(p.x, fq::sqr(p.zz)));
    r.y = fq::reduce_full(fq::mul(p.y, fq::sqr(p.zzz)));
    r.z = fq::reduce_full(p.zzz);
    return r;
  }
};

} // namespace bn254
