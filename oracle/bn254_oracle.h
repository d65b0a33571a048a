/*
 * CPU oracle for the BN254 G1 multi-scalar multiplication path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker
 * (or as the timed CPU baseline).  The product library never links it.
 *
 * It restates, in plain C with 4 x 64-bit limbs, the arithmetic that the
 * reference performs on the host and on the device:
 *   - Fq / Fr Montgomery arithmetic with R = 2^256
 *       (reference: src/ff_dispatch_st.cuh:485-508 host CIOS mul,
 *        :528 from_montgomery, :604-609 neg, :654-685 inverse;
 *        constants src/ff_config.cuh:7-84)
 *   - Jacobian doubling / addition used by the caller-side final reduction
 *       (src/ec.cuh:284-371, dbl-2009-l and add-2007-bl)
 *   - XYZZ mixed addition / addition / doubling used for bucket sums
 *       (src/ec.cuh:416-602, madd-2008-s, add-2008-s, dbl-2008-s-1)
 *   - the 254-point Horner reduction documented for msm_execute_async
 *       (src/bellman-cuda.h:496-505, tests/msm_test.cu:116-126)
 *   - the checksum oracle of the reference MSM test: when P_i = k_i * G the
 *       MSM equals (sum_i k_i * s_i mod r) * G (tests/msm_test.cu:27-32, 107-114)
 *   - a multithreaded host Pippenger (the timed CPU baseline).
 *
 * All buffers use the reference's byte layout: a field element is 8 x u32
 * little-endian limbs (32 bytes); an affine point is x then y (64 bytes); a
 * Jacobian point is x, y, z (96 bytes).  "mont" means Montgomery form.
 */
#ifndef BN254_ORACLE_H
#define BN254_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field helpers (p = base field Fq, r = scalar field Fr). */
void orc_fq_mul(const uint32_t a[8], const uint32_t b[8], uint32_t out[8]);
void orc_fq_to_mont(const uint32_t a[8], uint32_t out[8]);
void orc_fq_from_mont(const uint32_t a[8], uint32_t out[8]);
void orc_fr_to_mont(const uint32_t a[8], uint32_t out[8]);
void orc_fr_from_mont(const uint32_t a[8], uint32_t out[8]);
void orc_fr_to_mont_batch(const uint32_t *a, uint32_t *out, size_t n);

/* k * G for each standard-form scalar k (k < r); writes Montgomery-form affine
 * points (64 B each).  k == 0 is rejected (returns -1): affine has no infinity. */
int orc_gen_bases(const uint32_t *k_std, size_t n, uint32_t *bases_mont, int threads);

/* Normalised output: out_std[16] = affine (x, y) in standard form, fully
 * reduced; return value 1 = point at infinity (out zeroed), 0 = finite. */

/* sum_i s_i * P_i by double-and-add per term (slow, small n only). */
int orc_msm_naive(const uint32_t *bases_mont, const uint32_t *scalars_mont, size_t n, uint32_t out_std[16]);

/* Multithreaded Pippenger (signed windows, XYZZ buckets). threads <= 0: all cores. */
int orc_msm_pippenger(const uint32_t *bases_mont, const uint32_t *scalars_mont, size_t n, int threads, uint32_t out_std[16]);

/* (sum_i k_i * s_i mod r) * G, with k_std standard form and scalars Montgomery form. */
int orc_msm_checksum(const uint32_t *k_std, const uint32_t *scalars_mont, size_t n, uint32_t out_std[16]);

/* Horner reduction of `count` Montgomery Jacobian points: sum_i 2^i * R_i. */
int orc_horner(const uint32_t *results_jac_mont, size_t count, uint32_t out_std[16]);

/* Normalise one Montgomery Jacobian point. */
int orc_jacobian_normalize(const uint32_t jac_mont[24], uint32_t out_std[16]);

/* Affine point (Montgomery form) on the curve y^2 = x^3 + 3 ? */
int orc_affine_is_on_curve(const uint32_t aff_mont[16]);

/* Scalar multiple of a standard-form affine point, output standard affine. */
int orc_affine_mul(const uint32_t aff_std[16], const uint32_t k_std[8], uint32_t out_std[16]);

/* Point addition of two standard-form affine points (either may be flagged infinite). */
int orc_affine_add(const uint32_t a_std[16], int a_inf, const uint32_t b_std[16], int b_inf, uint32_t out_std[16]);

#ifdef __cplusplus
}
#endif

#endif
