// Thin C-ABI shim over the reference's OWN host-side field and curve code
// (src/ff_dispatch_st.cuh host branches, src/ec.cuh), compiled as host code by
// nvcc from the reference source tree (see oracle/Makefile, target `ref`).
// TEST INFRASTRUCTURE ONLY: the CPU tests use it to pin the C restatement in
// bn254_oracle.c against the reference itself.  Nothing here runs on a GPU.
#include "ec.cuh"
#include "ff_dispatch_st.cuh"
#include <cstdint>
#include <cstring>

// The template arguments name inv_p / inv_q (src/ff_config.cuh:37, :83); their
// definitions come from the reference's src/ff_config.cu, linked in by the
// Makefile with relocatable device code.

typedef fd_p fp;
typedef fd_q fq;
typedef ec<fp, 3> curve;
typedef curve::point_affine pa;
typedef curve::point_jacobian pj;
typedef curve::point_xyzz pz;

template <class T> static T load(const uint32_t *w) {
  T t;
  std::memcpy(&t, w, sizeof(T));
  return t;
}
template <class T> static void store(uint32_t *w, const T &t) { std::memcpy(w, &t, sizeof(T)); }

extern "C" {

void ref_fq_mul(const uint32_t *a, const uint32_t *b, uint32_t *out) {
  store(out, fp::mul(load<fp::storage>(a), load<fp::storage>(b)));
}

void ref_fq_to_mont(const uint32_t *a, uint32_t *out) { store(out, fp::to_montgomery(load<fp::storage>(a))); }

void ref_fq_from_mont(const uint32_t *a, uint32_t *out) { store(out, fp::from_montgomery(load<fp::storage>(a))); }

void ref_fr_to_mont(const uint32_t *a, uint32_t *out) { store(out, fq::to_montgomery(load<fq::storage>(a))); }

void ref_fr_from_mont(const uint32_t *a, uint32_t *out) { store(out, fq::from_montgomery(load<fq::storage>(a))); }

void ref_fq_inverse(const uint32_t *a, uint32_t *out) { store(out, fp::inverse(load<fp::storage>(a))); }

// XYZZ accumulator += affine base (madd-2008-s, host branch of src/ec.cuh:555-597)
void ref_xyzz_madd(const uint32_t *acc, const uint32_t *base, uint32_t *out) {
  store(out, curve::add(load<pz>(acc), load<pa>(base), fp()));
}

// XYZZ + XYZZ (add-2008-s, src/ec.cuh:495-546)
void ref_xyzz_add(const uint32_t *a, const uint32_t *b, uint32_t *out) { store(out, curve::add(load<pz>(a), load<pz>(b), fp())); }

// XYZZ -> Jacobian (src/ec.cuh:255-263)
void ref_xyzz_to_jacobian(const uint32_t *a, uint32_t *out) { store(out, pz::to_jacobian(load<pz>(a), fp())); }

// The caller-side Horner reduction of the 254 results (src/bellman-cuda.h:496-505),
// returning the Jacobian sum (Montgomery form).
void ref_horner(const uint32_t *results, unsigned count, uint32_t *out) {
  fp d;
  pj sum = pj::point_at_infinity(d);
  for (unsigned i = 0; i < count; i++) {
    unsigned index = count - i - 1;
    pj bucket = load<pj>(results + 24 * index);
    sum = i == 0 ? bucket : curve::add(curve::dbl(sum, d), bucket, d);
  }
  store(out, sum);
}

// scalar (standard form Fr) times a Montgomery affine point, via the reference's
// double-and-add (src/ec.cuh:764-790); Jacobian Montgomery output.
void ref_mul(const uint32_t *scalar, const uint32_t *base, uint32_t *out) {
  fp d;
  pj p = pa::to_jacobian(load<pa>(base), d);
  store(out, curve::mul<fq>(load<fq::storage>(scalar), p, d));
}

// sum_i s_i * P_i with the reference's host routines only: scalars converted
// from Montgomery form (src/ff_dispatch_st.cuh:528), each term by
// double-and-add (src/ec.cuh:764-790), summed with add-2007-bl.
void ref_msm_naive(const uint32_t *bases, const uint32_t *scalars, unsigned n, uint32_t *out) {
  fp d;
  pj sum = pj::point_at_infinity(d);
  for (unsigned i = 0; i < n; i++) {
    const fq::storage s = fq::from_montgomery(load<fq::storage>(scalars + 8 * i));
    const pj p = pa::to_jacobian(load<pa>(bases + 16 * i), d);
    sum = curve::add(sum, curve::mul<fq>(s, p, d), d);
  }
  store(out, sum);
}

// Jacobian equality up to projective scaling (src/ec.cuh:159-173).
int ref_jacobian_eq(const uint32_t *a, const uint32_t *b) { return pj::eq(load<pj>(a), load<pj>(b), fp()) ? 1 : 0; }

} // extern "C"
