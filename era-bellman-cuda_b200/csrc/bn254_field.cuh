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
#else
#define BN_HD inline
#define BN_DEV inline
#define BN_ALIGN(n) alignas(n)
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

  // ---- Montgomery multiplication (CIOS, one operand word per round) -------
  // Round i: T += a*b[i]  (low halves into words 0..7, high halves into 1..8),
  //          q = T[0]*INV,  T += q*m  (same two chains),  T >>= 32.
  // T < 2m*2^32 + 2m + m*2^32 < 2^288 during a round, so nine words hold it
  // and the last instruction of each high-half chain has no carry out.
  // 33 multiply instructions per round, 264 in total; inputs < 2m give an
  // output < 2m.
  static BN_HD fe mul(const fe &a, const fe &b) {
    uint32_t t0, t1, t2, t3, t4, t5, t6, t7, t8;
    // round 0: T = a*b[0] + q*m with T starting at zero
    {
      const uint32_t bi = b.l[0];
      t0 = cc::mul_lo(a.l[0], bi);
      t1 = cc::mul_lo(a.l[1], bi);
      t2 = cc::mul_lo(a.l[2], bi);
      t3 = cc::mul_lo(a.l[3], bi);
      t4 = cc::mul_lo(a.l[4], bi);
      t5 = cc::mul_lo(a.l[5], bi);
      t6 = cc::mul_lo(a.l[6], bi);
      t7 = cc::mul_lo(a.l[7], bi);
      t1 = cc::mad_hi_cc(a.l[0], bi, t1);
      t2 = cc::madc_hi_cc(a.l[1], bi, t2);
      t3 = cc::madc_hi_cc(a.l[2], bi, t3);
      t4 = cc::madc_hi_cc(a.l[3], bi, t4);
      t5 = cc::madc_hi_cc(a.l[4], bi, t5);
      t6 = cc::madc_hi_cc(a.l[5], bi, t6);
      t7 = cc::madc_hi_cc(a.l[6], bi, t7);
      t8 = cc::madc_hi(a.l[7], bi, 0);
      reduce_round(t0, t1, t2, t3, t4, t5, t6, t7, t8);
    }
#pragma unroll
    for (int i = 1; i < 8; i++) {
      const uint32_t bi = b.l[i];
      // t0..t7 hold T (< 2m), t8 == 0
      t0 = cc::mad_lo_cc(a.l[0], bi, t0);
      t1 = cc::madc_lo_cc(a.l[1], bi, t1);
      t2 = cc::madc_lo_cc(a.l[2], bi, t2);
      t3 = cc::madc_lo_cc(a.l[3], bi, t3);
      t4 = cc::madc_lo_cc(a.l[4], bi, t4);
      t5 = cc::madc_lo_cc(a.l[5], bi, t5);
      t6 = cc::madc_lo_cc(a.l[6], bi, t6);
      t7 = cc::madc_lo_cc(a.l[7], bi, t7);
      t8 = cc::addc(0, 0);
      t1 = cc::mad_hi_cc(a.l[0], bi, t1);
      t2 = cc::madc_hi_cc(a.l[1], bi, t2);
      t3 = cc::madc_hi_cc(a.l[2], bi, t3);
      t4 = cc::madc_hi_cc(a.l[3], bi, t4);
      t5 = cc::madc_hi_cc(a.l[4], bi, t5);
      t6 = cc::madc_hi_cc(a.l[5], bi, t6);
      t7 = cc::madc_hi_cc(a.l[6], bi, t7);
      t8 = cc::madc_hi(a.l[7], bi, t8);
      reduce_round(t0, t1, t2, t3, t4, t5, t6, t7, t8);
    }
    fe r;
    r.l[0] = t0;
    r.l[1] = t1;
    r.l[2] = t2;
    r.l[3] = t3;
    r.l[4] = t4;
    r.l[5] = t5;
    r.l[6] = t6;
    r.l[7] = t7;
    return r;
  }

  // One reduction round on the nine-word window t0..t8:
  //   q = t0*INV; (t0..t8) += q*m; shift down one word (t8 becomes 0).
  static BN_HD void reduce_round(uint32_t &t0, uint32_t &t1, uint32_t &t2, uint32_t &t3, uint32_t &t4, uint32_t &t5, uint32_t &t6,
                                 uint32_t &t7, uint32_t &t8) {
    const uint32_t q = cc::mul_lo(t0, F::INV);
    t0 = cc::mad_lo_cc(q, F::mod(0), t0); // == 0, only the carry matters
    t1 = cc::madc_lo_cc(q, F::mod(1), t1);
    t2 = cc::madc_lo_cc(q, F::mod(2), t2);
    t3 = cc::madc_lo_cc(q, F::mod(3), t3);
    t4 = cc::madc_lo_cc(q, F::mod(4), t4);
    t5 = cc::madc_lo_cc(q, F::mod(5), t5);
    t6 = cc::madc_lo_cc(q, F::mod(6), t6);
    t7 = cc::madc_lo_cc(q, F::mod(7), t7);
    t8 = cc::addc(t8, 0);
    t1 = cc::mad_hi_cc(q, F::mod(0), t1);
    t2 = cc::madc_hi_cc(q, F::mod(1), t2);
    t3 = cc::madc_hi_cc(q, F::mod(2), t3);
    t4 = cc::madc_hi_cc(q, F::mod(3), t4);
    t5 = cc::madc_hi_cc(q, F::mod(4), t5);
    t6 = cc::madc_hi_cc(q, F::mod(5), t6);
    t7 = cc::madc_hi_cc(q, F::mod(6), t7);
    t8 = cc::madc_hi(q, F::mod(7), t8);
    t0 = t1;
    t1 = t2;
    t2 = t3;
    t3 = t4;
    t4 = t5;
    t5 = t6;
    t6 = t7;
    t7 = t8;
    t8 = 0;
  }

  // Full 512-bit product (128 multiply instructions).  Row i adds a*b[i] at
  // word i; after row i the partial product is < 2^(32(i+9)), so the high
  // chain of row i never carries past word i+8.
  static BN_HD fe_wide mul_wide(const fe &a, const fe &b) {
    fe_wide w;
    {
      const uint32_t b0 = b.l[0];
#pragma unroll
      for (int j = 0; j < 8; j++)
        w.l[j] = cc::mul_lo(a.l[j], b0);
      w.l[1] = cc::mad_hi_cc(a.l[0], b0, w.l[1]);
#pragma unroll
      for (int j = 1; j < 7; j++)
        w.l[j + 1] = cc::madc_hi_cc(a.l[j], b0, w.l[j + 1]);
      w.l[8] = cc::madc_hi(a.l[7], b0, 0);
    }
#pragma unroll
    for (int i = 1; i < 8; i++) {
      const uint32_t bi = b.l[i];
      w.l[i] = cc::mad_lo_cc(a.l[0], bi, w.l[i]);
#pragma unroll
      for (int j = 1; j < 8; j++)
        w.l[i + j] = cc::madc_lo_cc(a.l[j], bi, w.l[i + j]);
      w.l[i + 8] = cc::addc(0, 0);
      w.l[i + 1] = cc::mad_hi_cc(a.l[0], bi, w.l[i + 1]);
#pragma unroll
      for (int j = 1; j < 7; j++)
        w.l[i + j + 1] = cc::madc_hi_cc(a.l[j], bi, w.l[i + j + 1]);
      w.l[i + 8] = cc::madc_hi(a.l[7], bi, w.l[i + 8]);
    }
    return w;
  }

  // 512-bit square: off-diagonal products once (56 instructions), doubled,
  // plus the diagonal (16 instructions).  Row i adds a[i]*a[j>i] at word i+j.
  static BN_HD fe_wide sqr_wide(const fe &a) {
    fe_wide w;
    w.l[0] = 0;
    // row 0: a0 * a1..a7 at words 1..8
    {
      const uint32_t ai = a.l[0];
#pragma unroll
      for (int j = 1; j < 8; j++)
        w.l[j] = cc::mul_lo(ai, a.l[j]);
      w.l[2] = cc::mad_hi_cc(ai, a.l[1], w.l[2]);
#pragma unroll
      for (int j = 2; j < 7; j++)
        w.l[j + 1] = cc::madc_hi_cc(ai, a.l[j], w.l[j + 1]);
      w.l[8] = cc::madc_hi(ai, a.l[7], 0);
    }
#pragma unroll
    for (int i = 1; i < 7; i++) {
      const uint32_t ai = a.l[i];
      // low halves of a[i]*a[j], j = i+1..7, at words 2i+1 .. i+7
      w.l[2 * i + 1] = cc::mad_lo_cc(ai, a.l[i + 1], w.l[2 * i + 1]);
#pragma unroll
      for (int j = i + 2; j < 8; j++)
        w.l[i + j] = cc::madc_lo_cc(ai, a.l[j], w.l[i + j]);
      w.l[i + 8] = cc::addc(0, 0);
      // high halves at words 2i+2 .. i+8
      if (i + 1 < 7) {
        w.l[2 * i + 2] = cc::mad_hi_cc(ai, a.l[i + 1], w.l[2 * i + 2]);
#pragma unroll
        for (int j = i + 2; j < 7; j++)
          w.l[i + j + 1] = cc::madc_hi_cc(ai, a.l[j], w.l[i + j + 1]);
        w.l[i + 8] = cc::madc_hi(ai, a.l[7], w.l[i + 8]);
      } else {
        // i == 6: the single product a6*a7
        w.l[14] = cc::mad_hi_cc(ai, a.l[7], w.l[14]);
      }
    }
    w.l[15] = 0;
    // double: shift the 512-bit off-diagonal sum left by one bit
    w.l[15] = (w.l[15] << 1) | (w.l[14] >> 31);
#pragma unroll
    for (int k = 14; k > 0; k--)
      w.l[k] = (w.l[k] << 1) | (w.l[k - 1] >> 31);
    w.l[0] = w.l[0] << 1;
    // add the diagonal a[i]^2 at words 2i, 2i+1
    w.l[0] = cc::mad_lo_cc(a.l[0], a.l[0], w.l[0]);
    w.l[1] = cc::madc_hi_cc(a.l[0], a.l[0], w.l[1]);
#pragma unroll
    for (int i = 1; i < 7; i++) {
      w.l[2 * i] = cc::madc_lo_cc(a.l[i], a.l[i], w.l[2 * i]);
      w.l[2 * i + 1] = cc::madc_hi_cc(a.l[i], a.l[i], w.l[2 * i + 1]);
    }
    w.l[14] = cc::madc_lo_cc(a.l[7], a.l[7], w.l[14]);
    w.l[15] = cc::madc_hi(a.l[7], a.l[7], w.l[15]);
    return w;
  }

  // Montgomery reduction of a 512-bit value w < m*2^256:
  // REDC(w) = REDC(w_lo) + w_hi, where REDC(w_lo) <= m; the result is < 2m
  // whenever w_hi < m (true for w < 4m^2).  136 multiply instructions.
  static BN_HD fe redc_wide(const fe_wide &w) {
    uint32_t t0 = w.l[0], t1 = w.l[1], t2 = w.l[2], t3 = w.l[3], t4 = w.l[4], t5 = w.l[5], t6 = w.l[6], t7 = w.l[7], t8 = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
      reduce_round(t0, t1, t2, t3, t4, t5, t6, t7, t8);
    fe r;
    r.l[0] = cc::add_cc(t0, w.l[8]);
    r.l[1] = cc::addc_cc(t1, w.l[9]);
    r.l[2] = cc::addc_cc(t2, w.l[10]);
    r.l[3] = cc::addc_cc(t3, w.l[11]);
    r.l[4] = cc::addc_cc(t4, w.l[12]);
    r.l[5] = cc::addc_cc(t5, w.l[13]);
    r.l[6] = cc::addc_cc(t6, w.l[14]);
    r.l[7] = cc::addc(t7, w.l[15]);
    return r;
  }

  static BN_HD fe sqr(const fe &a) { return redc_wide(sqr_wide(a)); }

  // a*b - c*d with one reduction: both products < 4m^2; a negative
  // difference is lifted by 4m^2, so the reduced operand is in [0, 4m^2).
  static BN_HD fe mul_sub_mul(const fe &a, const fe &b, const fe &c, const fe &d) {
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
  static BN_HD fe from_mont(const fe &a) {
    uint32_t t0 = a.l[0], t1 = a.l[1], t2 = a.l[2], t3 = a.l[3], t4 = a.l[4], t5 = a.l[5], t6 = a.l[6], t7 = a.l[7], t8 = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
      reduce_round(t0, t1, t2, t3, t4, t5, t6, t7, t8);
    fe r;
    r.l[0] = t0;
    r.l[1] = t1;
    r.l[2] = t2;
    r.l[3] = t3;
    r.l[4] = t4;
    r.l[5] = t5;
    r.l[6] = t6;
    r.l[7] = t7;
    return reduce_full(r);
  }

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
