// BN254 field core: 254-bit Montgomery arithmetic with 8 x 32-bit limbs.
//
// Fq (base field, p) and Fr (scalar field, r) share one implementation,
// parameterised by a constants struct.  R = 2^256 (the reference's choice,
// src/ff_config.cuh:7-84, so Montgomery-form inputs and outputs are
// byte-compatible with era-bellman-cuda).
//
// Value ranges ("lazy reduction"): both moduli are < 2^254, so 4m < 2^256 and
// every function below accepts and returns values in [0, 2m) unless stated.
// A Montgomery product of two values < 2m is < 2m without a final subtraction
// (a*b < 4m^2 < m*2^256), so no multiplication ends in a conditional subtract.
// Canonical [0, m) values are produced only by reduce_full(), for output.
//
// Carry handling: every multi-word operation is a sequence of single PTX
// carry-chain instructions (add.cc / addc / mad.lo.cc / madc.hi.cc ...).  On
// the host the same sequences run against an emulated carry flag, so the
// exact instruction order of every algorithm is exercised by CPU tests.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define BN_HD __host__ __device__ __forceinline__
#define BN_DEV __device__ __forceinline__
#define BN_ALIGN(n) __align__(n)
// rarely taken paths (point doubling inside an addition) stay out of line so
// the hot loop's instructions fit the instruction cache
#define BN_HD_COLD __host__ __device__ __noinline__
#define BN_HD_MUL __host__ __device__ __forceinline__
#else
#define BN_HD inline
#define BN_DEV inline
#define BN_ALIGN(n) alignas(n)
#define BN_HD_COLD inline
#define BN_HD_MUL inline
#endif

namespace bn254 {

// ---------------------------------------------------------------------------
// Carry-chain primitives.  Device: one PTX instruction each (asm volatile keeps
// their order, so the condition-code carry is not disturbed between them).
// Host: the carry flag is a thread-local variable.
// ---------------------------------------------------------------------------
#if !defined(__CUDA_ARCH__)
inline thread_local uint32_t host_carry_flag = 0;
#endif

namespace cc {

BN_HD uint32_t add_cc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  uint64_t s = (uint64_t)a + b;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

BN_HD uint32_t addc_cc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  uint64_t s = (uint64_t)a + b + host_carry_flag;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

BN_HD uint32_t addc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  return (uint32_t)((uint64_t)a + b + host_carry_flag);
#endif
}

BN_HD uint32_t sub_cc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  uint64_t d = (uint64_t)a - b;
  host_carry_flag = (uint32_t)(d >> 63);
  return (uint32_t)d;
#endif
}

BN_HD uint32_t subc_cc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  uint64_t d = (uint64_t)a - b - host_carry_flag;
  host_carry_flag = (uint32_t)(d >> 63);
  return (uint32_t)d;
#endif
}

BN_HD uint32_t subc(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
#else
  return (uint32_t)((uint64_t)a - b - host_carry_flag);
#endif
}

// r = lo(a*b) + c, carry out
BN_HD uint32_t mad_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
#else
  uint64_t s = (uint64_t)(uint32_t)((uint64_t)a * b) + c;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

// r = lo(a*b) + c + carry, carry out
BN_HD uint32_t madc_lo_cc(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
#else
  uint64_t s = (uint64_t)(uint32_t)((uint64_t)a * b) + c + host_carry_flag;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

// r = hi(a*b) + c, carry out
BN_HD uint32_t mad_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
#else
  uint64_t s = (((uint64_t)a * b) >> 32) + c;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

// r = hi(a*b) + c + carry, carry out
BN_HD uint32_t madc_hi_cc(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
#else
  uint64_t s = (((uint64_t)a * b) >> 32) + c + host_carry_flag;
  host_carry_flag = (uint32_t)(s >> 32);
  return (uint32_t)s;
#endif
}

// r = hi(a*b) + c + carry (no carry out)
BN_HD uint32_t madc_hi(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
#else
  return (uint32_t)((((uint64_t)a * b) >> 32) + c + host_carry_flag);
#endif
}

BN_HD uint32_t mul_lo(uint32_t a, uint32_t b) { return a * b; }

BN_HD uint32_t mul_hi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

} // namespace cc

// ---------------------------------------------------------------------------
// Storage
// ---------------------------------------------------------------------------
struct BN_ALIGN(16) fe {
  uint32_t l[8];
};

struct fe_wide {
  uint32_t l[16];
};

// Field constants.  The moduli are the BN254 primes; the rest is derived from
// them (and checked against big-integer arithmetic by the CPU tests).
struct fq_params {
  // p = 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47
  static BN_HD constexpr uint32_t mod(int i) {
    constexpr uint32_t v[8] = {0xd87cfd47, 0x3c208c16, 0x6871ca8d, 0x97816a91, 0x8181585d, 0xb85045b6, 0xe131a029, 0x30644e72};
    return v[i];
  }
  static BN_HD constexpr uint32_t mod2(int i) {
    constexpr uint32_t v[8] = {0xb0f9fa8e, 0x7841182d, 0xd0e3951a, 0x2f02d522, 0x0302b0bb, 0x70a08b6d, 0xc2634053, 0x60c89ce5};
    return v[i];
  }
  // 4 p^2, the offset that makes a difference of two products non-negative
  static BN_HD constexpr uint32_t mod_sq4(int i) {
    constexpr uint32_t v[16] = {0x9d75a6c4, 0xed516288, 0x27ab0404, 0x98081cb4, 0xb65b2b72, 0x29406271, 0xe8490b21, 0x11a27a55,
                                           0xd31ace34, 0x9bb7e970, 0x58dd5818, 0xc02e1544, 0x0d234872, 0x6669bdf0, 0xd8f2fe71, 0x249712e1};
    return v[i];
  }
  static constexpr uint32_t INV = 0xe4866389; // -p^-1 mod 2^32
  static BN_HD constexpr uint32_t one_mont(int i) {
    constexpr uint32_t v[8] = {0xc58f0d9d, 0xd35d438d, 0xf5c70b3d, 0x0a78eb28, 0x7879462c, 0x666ea36f, 0x9a07df2f, 0x0e0a77c1};
    return v[i];
  }  // 2^256 mod p
  static BN_HD constexpr uint32_t r2(int i) {
    constexpr uint32_t v[8] = {0x538afa89, 0xf32cfc5b, 0xd44501fb, 0xb5e71911, 0x0a417ff6, 0x47ab1eff, 0xcab8351f, 0x06d89f71};
    return v[i];
  }   // 2^512 mod p
};

struct fr_params {
  // r = 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001
  static BN_HD constexpr uint32_t mod(int i) {
    constexpr uint32_t v[8] = {0xf0000001, 0x43e1f593, 0x79b97091, 0x2833e848, 0x8181585d, 0xb85045b6, 0xe131a029, 0x30644e72};
    return v[i];
  }
  static BN_HD constexpr uint32_t mod2(int i) {
    constexpr uint32_t v[8] = {0xe0000002, 0x87c3eb27, 0xf372e122, 0x5067d090, 0x0302b0ba, 0x70a08b6d, 0xc2634053, 0x60c89ce5};
    return v[i];
  }
  static BN_HD constexpr uint32_t mod_sq4(int i) {
    constexpr uint32_t v[16] = {0x80000004, 0x230fac9f, 0x72cd0000, 0x1fc9888f, 0xa326edff, 0xffa698b1, 0xa08776c3, 0x9b3865d7,
                                           0x1ed8bf9e, 0xb1dd49ed, 0x4de74f7c, 0x17dceec3, 0x0d234872, 0x6669bdf0, 0xd8f2fe71, 0x249712e1};
    return v[i];
  }
  static constexpr uint32_t INV = 0xefffffff; // -r^-1 mod 2^32
  static BN_HD constexpr uint32_t one_mont(int i) {
    constexpr uint32_t v[8] = {0x4ffffffb, 0xac96341c, 0x9f60cd29, 0x36fc7695, 0x7879462e, 0x666ea36f, 0x9a07df2f, 0x0e0a77c1};
    return v[i];
  }
  static BN_HD constexpr uint32_t r2(int i) {
    constexpr uint32_t v[8] = {0xae216da7, 0x1bb8e645, 0xe35c59e3, 0x53fe3ab1, 0x53bb8085, 0x8c49833d, 0x7f4e44a5, 0x0216d0b1};
    return v[i];
  }
};

// ---------------------------------------------------------------------------
// Arithmetic.  F is fq_params or fr_params.
// ---------------------------------------------------------------------------
template <class F> struct field {

  static BN_HD fe zero() {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++)
      r.l[i] = 0;
    return r;
  }

  static BN_HD fe one() {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++)
      r.l[i] = F::one_mont(i);
    return r;
  }

  static BN_HD fe modulus() {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++)
      r.l[i] = F::mod(i);
    return r;
  }

  // a + b for a, b < 2m: the sum (< 4m < 2^256) minus 2m when that does not borrow.
  static BN_HD fe add(const fe &a, const fe &b) {
    fe s, d;
    s.l[0] = cc::add_cc(a.l[0], b.l[0]);
#pragma unroll
    for (int i = 1; i < 7; i++)
      s.l[i] = cc::addc_cc(a.l[i], b.l[i]);
    s.l[7] = cc::addc(a.l[7], b.l[7]);
    d.l[0] = cc::sub_cc(s.l[0], F::mod2(0));
#pragma unroll
    for (int i = 1; i < 8; i++)
      d.l[i] = cc::subc_cc(s.l[i], F::mod2(i));
    const uint32_t borrow = cc::subc(0, 0); // 0xffffffff when s < 2m
#pragma unroll
    for (int i = 0; i < 8; i++)
      d.l[i] = borrow ? s.l[i] : d.l[i];
    return d;
  }

  // a - b for a, b < 2m: wrap by adding 2m when the subtraction borrows.
  static BN_HD fe sub(const fe &a, const fe &b) {
    fe d;
    d.l[0] = cc::sub_cc(a.l[0], b.l[0]);
#pragma unroll
    for (int i = 1; i < 8; i++)
      d.l[i] = cc::subc_cc(a.l[i], b.l[i]);
    const uint32_t mask = cc::subc(0, 0); // all ones on borrow
    d.l[0] = cc::add_cc(d.l[0], F::mod2(0) & mask);
#pragma unroll
    for (int i = 1; i < 7; i++)
      d.l[i] = cc::addc_cc(d.l[i], F::mod2(i) & mask);
    d.l[7] = cc::addc(d.l[7], F::mod2(7) & mask);
    return d;
  }

  static BN_HD fe dbl(const fe &a) { return add(a, a); }

  static BN_HD fe neg(const fe &a) { return sub(zero(), a); }

  // 2m - a for a in (0, 2m): the negation of a nonzero value as a lazy value
  // in (0, 2m), one borrow chain
  static BN_HD fe neg_nonzero(const fe &a) {
    fe r;
    r.l[0] = cc::sub_cc(F::mod2(0), a.l[0]);
#pragma unroll
    for (int i = 1; i < 7; i++)
      r.l[i] = cc::subc_cc(F::mod2(i), a.l[i]);
    r.l[7] = cc::subc(F::mod2(7), a.l[7]);
    return r;
  }

  // [0, 2m) -> [0, m)
  static BN_HD fe reduce_full(const fe &a) {
    fe d;
    d.l[0] = cc::sub_cc(a.l[0], F::mod(0));
#pragma unroll
    for (int i = 1; i < 8; i++)
      d.l[i] = cc::subc_cc(a.l[i], F::mod(i));
    const uint32_t borrow = cc::subc(0, 0);
#pragma unroll
    for (int i = 0; i < 8; i++)
      d.l[i] = borrow ? a.l[i] : d.l[i];
    return d;
  }

  static BN_HD bool is_zero_exact(const fe &a) {
    uint32_t acc = a.l[0];
#pragma unroll
    for (int i = 1; i < 8; i++)
      acc |= a.l[i];
    return acc == 0;
  }

  // a in [0, 2m) is congruent to zero iff a == 0 or a == m.
  static BN_HD bool is_zero(const fe &a) {
    uint32_t z = a.l[0], m = a.l[0] ^ F::mod(0);
#pragma unroll
    for (int i = 1; i < 8; i++) {
      z |= a.l[i];
      m |= a.l[i] ^ F::mod(i);
    }
    return z == 0 || m == 0;
  }

  // ---- Montgomery multiplication -------------------------------------------
  // CIOS, one operand word per round.  T is held in two accumulators whose
  // words are used in fixed (low, high) pairs, so that the two halves of each
  // 32 x 32 product are adjacent in one carry chain and every pair keeps its
  // partner across rounds (a pair that changed partners would cost register
  // moves):
  //   the "even" accumulator takes products at word positions (0,1) (2,3)
  //   (4,5) (6,7) -- the even limbs x[0,2,4,6] times y, and q * m[0,2,4,6];
  //   the "odd" accumulator takes (1,2) (3,4) (5,6) (7,8) -- the odd limbs.
  // Dividing T by 2^32 moves every word down one position, which turns the
  // odd accumulator's pairs into even-aligned pairs and vice versa, so the
  // two arrays simply swap roles each round; array index = position + round.
  // The one word left unpaired (the old even accumulator's word at the new
  // position 0) is folded into the new even accumulator at the start of the
  // next round; its carry enters the odd chain, which starts at position 1.
  // During a round T < 4m + 3m * 2^32 < 2^288 and each accumulator is <= T,
  // so nine words hold either one and odd chains never carry out of their
  // last word.  33 multiply instructions per round; inputs < 2m give an
  // output < 2m.

  // A[R..R+7] += x[0,2,4,6] * y; carry into A[R+8] (fresh word)
  template <int R> static BN_HD void even_products(uint32_t *A, const uint32_t *x, uint32_t y) {
    A[R + 0] = cc::mad_lo_cc(x[0], y, A[R + 0]);
    A[R + 1] = cc::madc_hi_cc(x[0], y, A[R + 1]);
    A[R + 2] = cc::madc_lo_cc(x[2], y, A[R + 2]);
    A[R + 3] = cc::madc_hi_cc(x[2], y, A[R + 3]);
    A[R + 4] = cc::madc_lo_cc(x[4], y, A[R + 4]);
    A[R + 5] = cc::madc_hi_cc(x[4], y, A[R + 5]);
    A[R + 6] = cc::madc_lo_cc(x[6], y, A[R + 6]);
    A[R + 7] = cc::madc_hi_cc(x[6], y, A[R + 7]);
    A[R + 8] = cc::addc(A[R + 8], 0);
  }

  // B[R+1..R+8] += x[1,3,5,7] * y, no carry out; CARRY_IN consumes the flag
  template <int R, bool CARRY_IN> static BN_HD void odd_products(uint32_t *B, const uint32_t *x, uint32_t y) {
    B[R + 1] = CARRY_IN ? cc::madc_lo_cc(x[1], y, B[R + 1]) : cc::mad_lo_cc(x[1], y, B[R + 1]);
    B[R + 2] = cc::madc_hi_cc(x[1], y, B[R + 2]);
    B[R + 3] = cc::madc_lo_cc(x[3], y, B[R + 3]);
    B[R + 4] = cc::madc_hi_cc(x[3], y, B[R + 4]);
    B[R + 5] = cc::madc_lo_cc(x[5], y, B[R + 5]);
    B[R + 6] = cc::madc_hi_cc(x[5], y, B[R + 6]);
    B[R + 7] = cc::madc_lo_cc(x[7], y, B[R + 7]);
    B[R + 8] = cc::madc_hi(x[7], y, B[R + 8]);
  }

  // the same two chains against the modulus
  template <int R> static BN_HD void even_reduce(uint32_t *A, uint32_t q) {
    A[R + 0] = cc::mad_lo_cc(q, F::mod(0), A[R + 0]); // becomes 0; the carry matters
    A[R + 1] = cc::madc_hi_cc(q, F::mod(0), A[R + 1]);
    A[R + 2] = cc::madc_lo_cc(q, F::mod(2), A[R + 2]);
    A[R + 3] = cc::madc_hi_cc(q, F::mod(2), A[R + 3]);
    A[R + 4] = cc::madc_lo_cc(q, F::mod(4), A[R + 4]);
    A[R + 5] = cc::madc_hi_cc(q, F::mod(4), A[R + 5]);
    A[R + 6] = cc::madc_lo_cc(q, F::mod(6), A[R + 6]);
    A[R + 7] = cc::madc_hi_cc(q, F::mod(6), A[R + 7]);
    A[R + 8] = cc::addc(A[R + 8], 0);
  }

  template <int R, bool CARRY_IN> static BN_HD void odd_reduce(uint32_t *B, uint32_t q) {
    B[R + 1] = CARRY_IN ? cc::madc_lo_cc(q, F::mod(1), B[R + 1]) : cc::mad_lo_cc(q, F::mod(1), B[R + 1]);
    B[R + 2] = cc::madc_hi_cc(q, F::mod(1), B[R + 2]);
    B[R + 3] = cc::madc_lo_cc(q, F::mod(3), B[R + 3]);
    B[R + 4] = cc::madc_hi_cc(q, F::mod(3), B[R + 4]);
    B[R + 5] = cc::madc_lo_cc(q, F::mod(5), B[R + 5]);
    B[R + 6] = cc::madc_hi_cc(q, F::mod(5), B[R + 6]);
    B[R + 7] = cc::madc_lo_cc(q, F::mod(7), B[R + 7]);
    B[R + 8] = cc::madc_hi(q, F::mod(7), B[R + 8]);
  }

  // Round R >= 1 of the product (A = even role, B = odd role this round).
  template <int R> static BN_HD void mul_round(uint32_t *A, uint32_t *B, const uint32_t *x, uint32_t y) {
    A[R] = cc::add_cc(A[R], B[R]); // fold B's unpaired word; the carry belongs to position 1
    odd_products<R, true>(B, x, y);
    even_products<R>(A, x, y);
    const uint32_t q = cc::mul_lo(A[R], F::INV);
    even_reduce<R>(A, q);
    odd_reduce<R, false>(B, q);
  }

  // Round R >= 1 of a reduction without products.
  template <int R> static BN_HD void redc_round(uint32_t *A, uint32_t *B) {
    A[R] = cc::add_cc(A[R], B[R]);
    const uint32_t q = cc::mul_lo(A[R], F::INV);
    odd_reduce<R, true>(B, q);
    even_reduce<R>(A, q);
  }

  // result positions 0..7 live at index 8 of both arrays after eight rounds
  static BN_HD fe merge8(const uint32_t *X, const uint32_t *Y) {
    fe r;
    r.l[0] = cc::add_cc(X[8], Y[8]);
#pragma unroll
    for (int k = 1; k < 7; k++)
      r.l[k] = cc::addc_cc(X[8 + k], Y[8 + k]);
    r.l[7] = cc::addc(X[15], Y[15]);
    return r;
  }

  static BN_HD_MUL fe mul(const fe &a, const fe &b) { return mul_cios(a, b); }

  static BN_HD_MUL fe mul_cios(const fe &a, const fe &b) {
    uint32_t X[17], Y[17];
#pragma unroll
    for (int k = 0; k < 17; k++) {
      X[k] = 0;
      Y[k] = 0;
    }
    {
      // round 0 on T = 0: products land in empty words (X even role, Y odd)
      const uint32_t y = b.l[0];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        X[2 * k] = cc::mul_lo(a.l[2 * k], y);
        X[2 * k + 1] = cc::mul_hi(a.l[2 * k], y);
        Y[2 * k + 1] = cc::mul_lo(a.l[2 * k + 1], y);
        Y[2 * k + 2] = cc::mul_hi(a.l[2 * k + 1], y);
      }
      const uint32_t q = cc::mul_lo(X[0], F::INV);
      even_reduce<0>(X, q);
      odd_reduce<0, false>(Y, q);
    }
    mul_round<1>(Y, X, a.l, b.l[1]);
    mul_round<2>(X, Y, a.l, b.l[2]);
    mul_round<3>(Y, X, a.l, b.l[3]);
    mul_round<4>(X, Y, a.l, b.l[4]);
    mul_round<5>(Y, X, a.l, b.l[5]);
    mul_round<6>(X, Y, a.l, b.l[6]);
    mul_round<7>(Y, X, a.l, b.l[7]);
    return merge8(X, Y);
  }

  // Montgomery reduction of a 256-bit value: eight rounds of q*m only.
  // Returns REDC(x) = x * 2^-256 mod m in [0, m] (x + q*m < 2^256 (1 + m)).
  static BN_HD fe redc_low(const fe &x) {
    uint32_t X[17], Y[17];
#pragma unroll
    for (int k = 0; k < 17; k++) {
      X[k] = k < 8 ? x.l[k < 8 ? k : 0] : 0;
      Y[k] = 0;
    }
    {
      const uint32_t q = cc::mul_lo(X[0], F::INV);
      even_reduce<0>(X, q);
      odd_reduce<0, false>(Y, q);
    }
    redc_round<1>(Y, X);
    redc_round<2>(X, Y);
    redc_round<3>(Y, X);
    redc_round<4>(X, Y);
    redc_round<5>(Y, X);
    redc_round<6>(X, Y);
    redc_round<7>(Y, X);
    return merge8(X, Y);
  }

  // Full 512-bit product a*b (128 multiply instructions).  A product
  // a[j]*b[i] lands at word position i + j: E collects the even positions
  // (pairs (2k, 2k+1)), O the odd ones (pairs (2k+1, 2k+2)), so pairs never
  // change partners between rows.  Row i's partial sum is < 2^(32(i+9)):
  // the chain that ends at word i+7 carries into a fresh word i+8, the one
  // that ends at word i+8 never carries out.
  static BN_HD fe_wide mul_wide(const fe &a, const fe &b) {
    uint32_t E[17], O[17];
#pragma unroll
    for (int k = 0; k < 17; k++) {
      E[k] = 0;
      O[k] = 0;
    }
    {
      const uint32_t y = b.l[0];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        E[2 * k] = cc::mul_lo(a.l[2 * k], y);
        E[2 * k + 1] = cc::mul_hi(a.l[2 * k], y);
        O[2 * k + 1] = cc::mul_lo(a.l[2 * k + 1], y);
        O[2 * k + 2] = cc::mul_hi(a.l[2 * k + 1], y);
      }
    }
    wide_row<1>(E, O, a.l, b.l[1]);
    wide_row<2>(E, O, a.l, b.l[2]);
    wide_row<3>(E, O, a.l, b.l[3]);
    wide_row<4>(E, O, a.l, b.l[4]);
    wide_row<5>(E, O, a.l, b.l[5]);
    wide_row<6>(E, O, a.l, b.l[6]);
    wide_row<7>(E, O, a.l, b.l[7]);
    fe_wide w;
    w.l[0] = cc::add_cc(E[0], O[0]);
#pragma unroll
    for (int k = 1; k < 15; k++)
      w.l[k] = cc::addc_cc(E[k], O[k]);
    w.l[15] = cc::addc(E[15], O[15]);
    return w;
  }

  // row I >= 1 of mul_wide: even I puts even limbs at even positions (E) and
  // odd limbs at odd positions (O); odd I the other way round
  template <int I> static BN_HD void wide_row(uint32_t *E, uint32_t *O, const uint32_t *x, uint32_t y) {
    if (I % 2 == 0) {
      even_products<I>(E, x, y);        // E[I..I+7], carry into E[I+8]
      odd_products<I, false>(O, x, y);  // O[I+1..I+8]
    } else {
      even_products<I>(O, x, y);        // x[0,2,4,6] at odd positions I..I+7, carry into O[I+8]
      odd_products<I, false>(E, x, y);  // x[1,3,5,7] at even positions I+1..I+8
    }
  }

  // 512-bit square: off-diagonal products a[i]*a[j] (i < j, 56 instructions)
  // split by the parity of i + j so every chain pairs low and high halves,
  // doubled, plus the diagonal a[i]^2 (16 instructions).  A chain of row i
  // ends at most at word i + 8 and its carry goes to a word no earlier row
  // has written.
  static BN_HD fe_wide sqr_wide(const fe &a) {
    uint32_t E[16], O[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      E[k] = 0;
      O[k] = 0;
    }
#pragma unroll
    for (int i = 0; i < 7; i++) {
      const uint32_t x = a.l[i];
      // i + j odd: j = i+1, i+3, ... -> O
      O[2 * i + 1] = cc::mad_lo_cc(x, a.l[i + 1], O[2 * i + 1]);
      O[2 * i + 2] = cc::madc_hi_cc(x, a.l[i + 1], O[2 * i + 2]);
#pragma unroll
      for (int j = i + 3; j < 8; j += 2) {
        O[i + j] = cc::madc_lo_cc(x, a.l[j], O[i + j]);
        O[i + j + 1] = cc::madc_hi_cc(x, a.l[j], O[i + j + 1]);
      }
      {
        const int last = i + 1 + 2 * ((7 - (i + 1)) / 2); // largest j of that parity
        O[i + last + 2] = cc::addc(O[i + last + 2], 0);
      }
      // i + j even: j = i+2, i+4, ... -> E
      if (i + 2 < 8) {
        E[2 * i + 2] = cc::mad_lo_cc(x, a.l[i + 2], E[2 * i + 2]);
        E[2 * i + 3] = cc::madc_hi_cc(x, a.l[i + 2], E[2 * i + 3]);
#pragma unroll
        for (int j = i + 4; j < 8; j += 2) {
          E[i + j] = cc::madc_lo_cc(x, a.l[j], E[i + j]);
          E[i + j + 1] = cc::madc_hi_cc(x, a.l[j], E[i + j + 1]);
        }
        const int last = i + 2 + 2 * ((7 - (i + 2)) / 2);
        E[i + last + 2] = cc::addc(E[i + last + 2], 0);
      }
    }
    // S = E + O (the off-diagonal sum, < 2^511), then 2S + diagonal
    uint32_t S[16];
    S[0] = cc::add_cc(E[0], O[0]);
#pragma unroll
    for (int k = 1; k < 15; k++)
      S[k] = cc::addc_cc(E[k], O[k]);
    S[15] = cc::addc(E[15], O[15]);
    fe_wide w;
    w.l[0] = cc::add_cc(S[0], S[0]);
#pragma unroll
    for (int k = 1; k < 15; k++)
      w.l[k] = cc::addc_cc(S[k], S[k]);
    w.l[15] = cc::addc(S[15], S[15]);
    w.l[0] = cc::mad_lo_cc(a.l[0], a.l[0], w.l[0]);
    w.l[1] = cc::madc_hi_cc(a.l[0], a.l[0], w.l[1]);
#pragma unroll
    for (int k = 1; k < 7; k++) {
      w.l[2 * k] = cc::madc_lo_cc(a.l[k], a.l[k], w.l[2 * k]);
      w.l[2 * k + 1] = cc::madc_hi_cc(a.l[k], a.l[k], w.l[2 * k + 1]);
    }
    w.l[14] = cc::madc_lo_cc(a.l[7], a.l[7], w.l[14]);
    w.l[15] = cc::madc_hi(a.l[7], a.l[7], w.l[15]);
    return w;
  }

  // Montgomery reduction of a 512-bit value w < m*2^256:
  // REDC(w) = REDC(w_lo) + w_hi with REDC(w_lo) <= m; the result is < 2m
  // whenever w_hi < m (true for w < 4m^2).  136 multiply instructions.
  static BN_HD fe redc_wide(const fe_wide &w) {
    fe lo;
#pragma unroll
    for (int k = 0; k < 8; k++)
      lo.l[k] = w.l[k];
    const fe r = redc_low(lo);
    fe out;
    out.l[0] = cc::add_cc(r.l[0], w.l[8]);
#pragma unroll
    for (int k = 1; k < 7; k++)
      out.l[k] = cc::addc_cc(r.l[k], w.l[k + 8]);
    out.l[7] = cc::addc(r.l[7], w.l[15]);
    return out;
  }

  static BN_HD_MUL fe sqr(const fe &a) { return redc_wide(sqr_wide(a)); }

  // a*b - c*d with one reduction: both products < 4m^2; a negative
  // difference is lifted by 4m^2, so the reduced operand is in [0, 4m^2).
  static BN_HD_MUL fe mul_sub_mul(const fe &a, const fe &b, const fe &c, const fe &d) {
    fe_wide x = mul_wide(a, b);
    const fe_wide y = mul_wide(c, d);
    x.l[0] = cc::sub_cc(x.l[0], y.l[0]);
#pragma unroll
    for (int i = 1; i < 16; i++)
      x.l[i] = cc::subc_cc(x.l[i], y.l[i]);
    const uint32_t mask = cc::subc(0, 0);
    x.l[0] = cc::add_cc(x.l[0], F::mod_sq4(0) & mask);
#pragma unroll
    for (int i = 1; i < 15; i++)
      x.l[i] = cc::addc_cc(x.l[i], F::mod_sq4(i) & mask);
    x.l[15] = cc::addc(x.l[15], F::mod_sq4(15) & mask);
    return redc_wide(x);
  }

  // Montgomery -> standard form, fully reduced.  Any 256-bit input works:
  // REDC(a) <= m, and a result equal to m folds to 0.
  static BN_HD fe from_mont(const fe &a) { return reduce_full(redc_low(a)); }

  // standard -> Montgomery form (input < 2m), fully reduced
  static BN_HD fe to_mont(const fe &a) {
    fe r2;
#pragma unroll
    for (int i = 0; i < 8; i++)
      r2.l[i] = F::r2(i);
    return reduce_full(mul(a, r2));
  }

  // a < b for canonical values
  static BN_HD bool lt(const fe &a, const fe &b) {
    uint32_t d = cc::sub_cc(a.l[0], b.l[0]);
#pragma unroll
    for (int i = 1; i < 8; i++)
      d = cc::subc_cc(a.l[i], b.l[i]);
    (void)d;
    return cc::subc(0, 0) != 0;
  }

  // ---- binary inversion (standard form) ------------------------------------
  static BN_HD bool is_one_raw(const fe &a) {
    uint32_t acc = a.l[0] ^ 1u;
#pragma unroll
    for (int i = 1; i < 8; i++)
      acc |= a.l[i];
    return acc == 0;
  }

  static BN_HD fe shr1(const fe &a, uint32_t top) {
    fe r;
#pragma unroll
    for (int i = 0; i < 7; i++)
      r.l[i] = (a.l[i] >> 1) | (a.l[i + 1] << 31);
    r.l[7] = (a.l[7] >> 1) | (top << 31);
    return r;
  }

  // a / 2 mod m for a canonical a: a >> 1, or (a + m) >> 1 for odd a (the
  // carry of a + m becomes bit 255)
  static BN_HD fe half_mod(const fe &a) {
    if (!(a.l[0] & 1))
      return shr1(a, 0);
    fe s;
    s.l[0] = cc::add_cc(a.l[0], F::mod(0));
#pragma unroll
    for (int i = 1; i < 8; i++)
      s.l[i] = cc::addc_cc(a.l[i], F::mod(i));
    return shr1(s, cc::addc(0, 0));
  }

  // a - b for a >= b
  static BN_HD fe sub_raw(const fe &a, const fe &b) {
    fe d;
    d.l[0] = cc::sub_cc(a.l[0], b.l[0]);
#pragma unroll
    for (int i = 1; i < 7; i++)
      d.l[i] = cc::subc_cc(a.l[i], b.l[i]);
    d.l[7] = cc::subc(a.l[7], b.l[7]);
    return d;
  }

  // a - b mod m for canonical a, b
  static BN_HD fe sub_canonical(const fe &a, const fe &b) {
    if (!lt(a, b))
      return sub_raw(a, b);
    fe s;
    s.l[0] = cc::add_cc(a.l[0], F::mod(0));
#pragma unroll
    for (int i = 1; i < 7; i++)
      s.l[i] = cc::addc_cc(a.l[i], F::mod(i));
    s.l[7] = cc::addc(a.l[7], F::mod(7));
    return sub_raw(s, b); // a + m - b < m, no wrap
  }

  // a^-1 mod m for a canonical a in standard (not Montgomery) form, by the
  // binary extended Euclidean algorithm (Hankerson, Menezes and Vanstone,
  // "Guide to Elliptic Curve Cryptography", Algorithm 2.22): with u = x1 a
  // and v = x2 a (mod m) kept invariant, halvings of the even one and the
  // subtraction of the smaller from the larger bring u or v to 1.  About
  // 2 x 254 rounds of shifts and subtractions: a much shorter dependent chain
  // than the 254 Montgomery squarings of the Fermat inverse, which is what a
  // single GPU thread finishing an MSM needs.  0 (and any a sharing a factor
  // with m) gives 0; every loop is bounded.
  static BN_HD fe inverse_binary(const fe &a) {
    fe u = a, v = modulus(), x1 = zero(), x2 = zero();
    x1.l[0] = 1;
    if (is_zero_exact(a))
      return zero();
    for (int round = 0; round < 1024; round++) {
      if (is_one_raw(u))
        return x1;
      if (is_one_raw(v))
        return x2;
      if (is_zero_exact(u) || is_zero_exact(v))
        break;
      while (!(u.l[0] & 1)) {
        u = shr1(u, 0);
        x1 = half_mod(x1);
      }
      while (!(v.l[0] & 1)) {
        v = shr1(v, 0);
        x2 = half_mod(x2);
      }
      if (!lt(u, v)) {
        u = sub_raw(u, v);
        x1 = sub_canonical(x1, x2);
      } else {
        v = sub_raw(v, u);
        x2 = sub_canonical(x2, x1);
      }
    }
    return zero();
  }

  // exponentiation by m - 2 (Fermat inverse), Montgomery domain; 0 -> 0
  static BN_HD fe inverse(const fe &a) {
    fe e = modulus();
    e.l[0] -= 2; // m is odd and > 2, no borrow
    fe acc = one();
    for (int i = 255; i >= 0; i--) {
      acc = sqr(acc);
      if ((e.l[i >> 5] >> (i & 31)) & 1)
        acc = mul(acc, a);
    }
    return acc;
  }
};

typedef field<fq_params> fq;
typedef field<fr_params> fr;

} // namespace bn254
