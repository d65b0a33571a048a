// CPU check of the product field / curve code (era-bellman-cuda_b200/csrc),
// compiled by g++ so that the carry-chain sequences run on the host against
// the emulated carry flag.  Test infrastructure: loaded by tests/ via ctypes.
#include "bn254_curve.cuh"

#include <cstring>

using namespace bn254;

template <class T> static T ld(const uint32_t *w) {
  T t;
  std::memcpy(&t, w, sizeof(T));
  return t;
}
template <class T> static void st(uint32_t *w, const T &t) { std::memcpy(w, &t, sizeof(T)); }

extern "C" {

// op: 0 mul, 1 sqr, 2 add, 3 sub, 4 neg, 5 reduce_full, 6 from_mont, 7 to_mont, 8 inverse, 9 dbl
void fc_fq_op(int op, const uint32_t *a, const uint32_t *b, uint32_t *out, int n) {
  for (int i = 0; i < n; i++) {
    const fe x = ld<fe>(a + 8 * i), y = ld<fe>(b + 8 * i);
    fe r{};
    switch (op) {
    case 0: r = fq::mul(x, y); break;
    case 1: r = fq::sqr(x); break;
    case 2: r = fq::add(x, y); break;
    case 3: r = fq::sub(x, y); break;
    case 4: r = fq::neg(x); break;
    case 5: r = fq::reduce_full(x); break;
    case 6: r = fq::from_mont(x); break;
    case 7: r = fq::to_mont(x); break;
    case 8: r = fq::inverse(x); break;
    case 9: r = fq::dbl(x); break;
    case 10: r = fq::neg_nonzero(x); break;
    case 11: r = fq::inverse_binary(x); break;
    }
    st(out + 8 * i, r);
  }
}

void fc_fr_op(int op, const uint32_t *a, const uint32_t *b, uint32_t *out, int n) {
  for (int i = 0; i < n; i++) {
    const fe x = ld<fe>(a + 8 * i), y = ld<fe>(b + 8 * i);
    fe r{};
    switch (op) {
    case 0: r = fr::mul(x, y); break;
    case 1: r = fr::sqr(x); break;
    case 6: r = fr::from_mont(x); break;
    case 7: r = fr::to_mont(x); break;
    }
    st(out + 8 * i, r);
  }
}

// a*b - c*d
void fc_fq_mul_sub_mul(const uint32_t *a, const uint32_t *b, const uint32_t *c, const uint32_t *d, uint32_t *out, int n) {
  for (int i = 0; i < n; i++)
    st(out + 8 * i, fq::mul_sub_mul(ld<fe>(a + 8 * i), ld<fe>(b + 8 * i), ld<fe>(c + 8 * i), ld<fe>(d + 8 * i)));
}

int fc_fq_is_zero(const uint32_t *a) { return fq::is_zero(ld<fe>(a)) ? 1 : 0; }

// 512-bit products (kind 0: schoolbook mul_wide, 2: sqr_wide) and Montgomery
// products (kind 3: CIOS, 5: sqr as mul_wide + REDC)
void fc_fq_wide(int kind, const uint32_t *a, const uint32_t *b, uint32_t *out, int n) {
  for (int i = 0; i < n; i++) {
    const fe x = ld<fe>(a + 8 * i), y = ld<fe>(b + 8 * i);
    switch (kind) {
    case 0: st(out + 16 * i, fq::mul_wide(x, y)); break;
    case 2: st(out + 16 * i, fq::sqr_wide(x)); break;
    case 3: st(out + 8 * i, fq::mul_cios(x, y)); break;
    case 5: st(out + 8 * i, fq::sqr(x)); break;
    }
  }
}

// curve: xyzz (32 words), affine (16 words), jacobian (24 words)
void fc_add_affine(const uint32_t *p, const uint32_t *a, uint32_t *out) { st(out, curve::add_affine(ld<xyzz>(p), ld<affine>(a))); }
int fc_add_affine_finite(const uint32_t *p, const uint32_t *a, uint32_t *out) {
  bool inf = false;
  st(out, curve::add_affine_finite(ld<xyzz>(p), ld<affine>(a), inf));
  return inf ? 1 : 0;
}
void fc_add(const uint32_t *p, const uint32_t *q, uint32_t *out) { st(out, curve::add(ld<xyzz>(p), ld<xyzz>(q))); }
void fc_dbl(const uint32_t *p, uint32_t *out) { st(out, curve::dbl(ld<xyzz>(p))); }
void fc_from_affine(const uint32_t *a, uint32_t *out) { st(out, curve::from_affine(ld<affine>(a))); }
void fc_to_jacobian(const uint32_t *p, uint32_t *out) { st(out, curve::to_jacobian(ld<xyzz>(p))); }
void fc_from_jacobian(const uint32_t *p, uint32_t *out) { st(out, curve::from_jacobian(ld<jacobian>(p))); }
int fc_to_affine_standard(const uint32_t *p, uint32_t *out) {
  fe x, y;
  const bool inf = curve::to_affine_standard(ld<xyzz>(p), x, y);
  st(out, x);
  st(out + 8, y);
  return inf ? 1 : 0;
}
void fc_infinity(uint32_t *out) { st(out, curve::infinity()); }

} // extern "C"
