/*
 * CPU oracle for the BN254 G1 MSM path -- TEST INFRASTRUCTURE ONLY (see
 * bn254_oracle.h for what may use it).  Plain C99 + unsigned __int128, 4 x u64
 * limbs, no dependencies besides pthreads.
 *
 * Each function names the reference code whose behaviour it restates
 * (paths relative to the era-bellman-cuda source tree).
 */
#include "bn254_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef unsigned __int128 u128;
typedef uint64_t u64;

/* ------------------------------------------------------------------------ */
/* Field parameters (values of src/ff_config.cuh:11 and :44; R = 2^256).      */
/* The derived constants (R mod m, R^2 mod m, -m^-1 mod 2^64) are computed at  */
/* start-up from the modulus so that no hand-typed derived value can be wrong. */
/* ------------------------------------------------------------------------ */
typedef struct {
  u64 m[4];
  u64 inv; /* -m^{-1} mod 2^64 */
  u64 one[4]; /* R mod m */
  u64 r2[4];  /* R^2 mod m */
} field;

static field FQ = {{0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {0}, {0}};
static field FR = {{0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {0}, {0}};

static int geq(const u64 a[4], const u64 b[4]) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] != b[i])
      return a[i] > b[i];
  }
  return 1;
}

static u64 add4(u64 r[4], const u64 a[4], const u64 b[4]) {
  u128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (u128)a[i] + b[i];
    r[i] = (u64)c;
    c >>= 64;
  }
  return (u64)c;
}

static u64 sub4(u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 borrow = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a[i] - b[i] - borrow;
    r[i] = (u64)d;
    borrow = (u64)(d >> 64) & 1;
  }
  return borrow;
}

static void f_add(const field *f, u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 t[4];
  u64 c = add4(t, a, b);
  if (c || geq(t, f->m))
    sub4(t, t, f->m);
  memcpy(r, t, sizeof t);
}

static void f_sub(const field *f, u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 t[4];
  if (sub4(t, a, b))
    add4(t, t, f->m);
  memcpy(r, t, sizeof t);
}

static void f_neg(const field *f, u64 r[4], const u64 a[4]) {
  static const u64 zero[4] = {0, 0, 0, 0};
  f_sub(f, r, zero, a);
}

/* Montgomery product a*b*2^-256 mod m by CIOS; inputs and output in [0, m).
 * (reference host path: src/ff_dispatch_st.cuh:485-508, 32-bit limbs there) */
static void f_mul(const field *f, u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 acc;
    u64 carry = 0;
    for (int j = 0; j < 4; j++) {
      acc = (u128)a[j] * b[i] + t[j] + carry;
      t[j] = (u64)acc;
      carry = (u64)(acc >> 64);
    }
    acc = (u128)t[4] + carry;
    t[4] = (u64)acc;
    t[5] = (u64)(acc >> 64);
    u64 q = t[0] * f->inv;
    acc = (u128)q * f->m[0] + t[0];
    carry = (u64)(acc >> 64);
    for (int j = 1; j < 4; j++) {
      acc = (u128)q * f->m[j] + t[j] + carry;
      t[j - 1] = (u64)acc;
      carry = (u64)(acc >> 64);
    }
    acc = (u128)t[4] + carry;
    t[3] = (u64)acc;
    t[4] = t[5] + (u64)(acc >> 64);
  }
  u64 res[4] = {t[0], t[1], t[2], t[3]};
  if (t[4] || geq(res, f->m))
    sub4(res, res, f->m);
  memcpy(r, res, sizeof res);
}

static void f_sqr(const field *f, u64 r[4], const u64 a[4]) { f_mul(f, r, a, a); }

static int f_is_zero(const u64 a[4]) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

static int f_eq(const u64 a[4], const u64 b[4]) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3]; }

static void f_to_mont(const field *f, u64 r[4], const u64 a[4]) {
  u64 t[4];
  memcpy(t, a, sizeof t);
  while (geq(t, f->m)) /* accept unreduced input, like mul by R^2 would */
    sub4(t, t, f->m);
  f_mul(f, r, t, f->r2);
}

/* reference: src/ff_dispatch_st.cuh:528 (multiply by the integer 1) */
static void f_from_mont(const field *f, u64 r[4], const u64 a[4]) {
  static const u64 one_int[4] = {1, 0, 0, 0};
  f_mul(f, r, a, one_int);
}

/* a^(m-2) in the Montgomery domain (Fermat); 0 maps to 0 like the reference's
 * binary-EEA inverse (src/ff_dispatch_st.cuh:654-685). */
static void f_inv(const field *f, u64 r[4], const u64 a[4]) {
  if (f_is_zero(a)) {
    memset(r, 0, 32);
    return;
  }
  u64 e[4];
  static const u64 two[4] = {2, 0, 0, 0};
  sub4(e, f->m, two);
  u64 acc[4];
  memcpy(acc, f->one, 32);
  for (int i = 255; i >= 0; i--) {
    f_sqr(f, acc, acc);
    if ((e[i / 64] >> (i % 64)) & 1)
      f_mul(f, acc, acc, a);
  }
  memcpy(r, acc, 32);
}

static void field_init(field *f) {
  /* -m^{-1} mod 2^64 by Newton iteration */
  u64 x = 1;
  for (int i = 0; i < 7; i++)
    x *= 2 - f->m[0] * x;
  f->inv = (u64)0 - x;
  /* R mod m: double 1 two hundred fifty-six times modulo m */
  u64 t[4] = {1, 0, 0, 0};
  for (int i = 0; i < 256; i++) {
    u64 c = add4(t, t, t);
    if (c || geq(t, f->m))
      sub4(t, t, f->m);
  }
  memcpy(f->one, t, 32);
  for (int i = 0; i < 256; i++) {
    u64 c = add4(t, t, t);
    if (c || geq(t, f->m))
      sub4(t, t, f->m);
  }
  memcpy(f->r2, t, 32);
}

static pthread_once_t init_once = PTHREAD_ONCE_INIT;
static void init_all(void) {
  field_init(&FQ);
  field_init(&FR);
}
#define INIT() pthread_once(&init_once, init_all)

static void load8(u64 r[4], const uint32_t *w) {
  for (int i = 0; i < 4; i++)
    r[i] = (u64)w[2 * i] | ((u64)w[2 * i + 1] << 32);
}

static void store8(uint32_t *w, const u64 a[4]) {
  for (int i = 0; i < 4; i++) {
    w[2 * i] = (uint32_t)a[i];
    w[2 * i + 1] = (uint32_t)(a[i] >> 32);
  }
}

/* ------------------------------------------------------------------------ */
/* Curve y^2 = x^3 + 3 over Fq, all coordinates in Montgomery form.          */
/* ------------------------------------------------------------------------ */
typedef struct {
  u64 x[4], y[4];
} aff;
typedef struct {
  u64 x[4], y[4], z[4];
} jac; /* x = X/Z^2, y = Y/Z^3; infinity iff Z == 0 */
typedef struct {
  u64 x[4], y[4], zz[4], zzz[4];
} xyzz; /* x = X/ZZ, y = Y/ZZZ; infinity iff ZZ == 0 */

static void jac_set_inf(jac *p) {
  memset(p, 0, sizeof *p);
  memcpy(p->y, FQ.one, 32);
}

static void xyzz_set_inf(xyzz *p) {
  memset(p, 0, sizeof *p);
  memcpy(p->y, FQ.one, 32);
}

/* dbl-2009-l (reference: src/ec.cuh:284-306) */
static void jac_dbl(jac *r, const jac *p) {
  if (f_is_zero(p->z)) {
    *r = *p;
    return;
  }
  const field *f = &FQ;
  u64 A[4], B[4], C[4], D[4], E[4], F[4], t[4], X3[4], Y3[4], Z3[4];
  f_sqr(f, A, p->x);
  f_sqr(f, B, p->y);
  f_sqr(f, C, B);
  f_add(f, t, p->x, B);
  f_sqr(f, t, t);
  f_sub(f, t, t, A);
  f_sub(f, t, t, C);
  f_add(f, D, t, t);
  f_add(f, E, A, A);
  f_add(f, E, E, A);
  f_sqr(f, F, E);
  f_sub(f, X3, F, D);
  f_sub(f, X3, X3, D);
  f_sub(f, t, D, X3);
  f_mul(f, Y3, E, t);
  f_add(f, t, C, C);
  f_add(f, t, t, t);
  f_add(f, t, t, t);
  f_sub(f, Y3, Y3, t);
  f_mul(f, Z3, p->y, p->z);
  f_add(f, Z3, Z3, Z3);
  memcpy(r->x, X3, 32);
  memcpy(r->y, Y3, 32);
  memcpy(r->z, Z3, 32);
}

/* add-2007-bl with the equal / opposite / infinity cases
 * (reference: src/ec.cuh:308-345) */
static void jac_add(jac *r, const jac *p, const jac *q) {
  if (f_is_zero(p->z)) {
    *r = *q;
    return;
  }
  if (f_is_zero(q->z)) {
    *r = *p;
    return;
  }
  const field *f = &FQ;
  u64 Z1Z1[4], Z2Z2[4], U1[4], U2[4], S1[4], S2[4], t[4];
  f_sqr(f, Z1Z1, p->z);
  f_sqr(f, Z2Z2, q->z);
  f_mul(f, U1, p->x, Z2Z2);
  f_mul(f, U2, q->x, Z1Z1);
  f_mul(f, t, q->z, Z2Z2);
  f_mul(f, S1, p->y, t);
  f_mul(f, t, p->z, Z1Z1);
  f_mul(f, S2, q->y, t);
  if (f_eq(U1, U2)) {
    if (f_eq(S1, S2)) {
      jac_dbl(r, p);
    } else {
      jac_set_inf(r);
    }
    return;
  }
  u64 H[4], I[4], J[4], rr[4], V[4], X3[4], Y3[4], Z3[4];
  f_sub(f, H, U2, U1);
  f_add(f, I, H, H);
  f_sqr(f, I, I);
  f_mul(f, J, H, I);
  f_sub(f, rr, S2, S1);
  f_add(f, rr, rr, rr);
  f_mul(f, V, U1, I);
  f_sqr(f, X3, rr);
  f_sub(f, X3, X3, J);
  f_sub(f, X3, X3, V);
  f_sub(f, X3, X3, V);
  f_sub(f, t, V, X3);
  f_mul(f, Y3, rr, t);
  f_mul(f, t, S1, J);
  f_add(f, t, t, t);
  f_sub(f, Y3, Y3, t);
  f_add(f, Z3, p->z, q->z);
  f_sqr(f, Z3, Z3);
  f_sub(f, Z3, Z3, Z1Z1);
  f_sub(f, Z3, Z3, Z2Z2);
  f_mul(f, Z3, Z3, H);
  memcpy(r->x, X3, 32);
  memcpy(r->y, Y3, 32);
  memcpy(r->z, Z3, 32);
}

/* mdbl-2008-s-1: doubling of an affine point into XYZZ (src/ec.cuh:416-445) */
static void xyzz_dbl_affine(xyzz *r, const aff *p) {
  const field *f = &FQ;
  u64 U[4], V[4], W[4], S[4], M[4], t[4];
  f_add(f, U, p->y, p->y);
  f_sqr(f, V, U);
  f_mul(f, W, U, V);
  f_mul(f, S, p->x, V);
  f_sqr(f, M, p->x);
  f_add(f, t, M, M);
  f_add(f, M, M, t);
  f_sqr(f, r->x, M);
  f_sub(f, r->x, r->x, S);
  f_sub(f, r->x, r->x, S);
  f_sub(f, t, S, r->x);
  f_mul(f, t, M, t);
  f_mul(f, r->y, W, p->y);
  f_sub(f, r->y, t, r->y);
  memcpy(r->zz, V, 32);
  memcpy(r->zzz, W, 32);
}

/* dbl-2008-s-1 (src/ec.cuh:450-487) */
static void xyzz_dbl(xyzz *r, const xyzz *p) {
  if (f_is_zero(p->zz)) {
    *r = *p;
    return;
  }
  const field *f = &FQ;
  u64 U[4], V[4], W[4], S[4], M[4], t[4], X3[4], Y3[4];
  f_add(f, U, p->y, p->y);
  f_sqr(f, V, U);
  f_mul(f, W, U, V);
  f_mul(f, S, p->x, V);
  f_sqr(f, M, p->x);
  f_add(f, t, M, M);
  f_add(f, M, M, t);
  f_sqr(f, X3, M);
  f_sub(f, X3, X3, S);
  f_sub(f, X3, X3, S);
  f_sub(f, t, S, X3);
  f_mul(f, t, M, t);
  f_mul(f, Y3, W, p->y);
  f_sub(f, Y3, t, Y3);
  f_mul(f, r->zz, V, p->zz);
  f_mul(f, r->zzz, W, p->zzz);
  memcpy(r->x, X3, 32);
  memcpy(r->y, Y3, 32);
}

/* madd-2008-s: XYZZ + affine with the infinity and equal-point cases
 * (src/ec.cuh:555-597) */
static void xyzz_madd(xyzz *r, const xyzz *p, const aff *q) {
  const field *f = &FQ;
  if (f_is_zero(p->zz)) {
    memcpy(r->x, q->x, 32);
    memcpy(r->y, q->y, 32);
    memcpy(r->zz, FQ.one, 32);
    memcpy(r->zzz, FQ.one, 32);
    return;
  }
  u64 U2[4], S2[4], P[4], R[4];
  f_mul(f, U2, q->x, p->zz);
  f_mul(f, S2, q->y, p->zzz);
  f_sub(f, P, U2, p->x);
  f_sub(f, R, S2, p->y);
  if (f_is_zero(P) && f_is_zero(R)) {
    xyzz_dbl_affine(r, q);
    return;
  }
  u64 PP[4], PPP[4], Q[4], X3[4], Y3[4], t[4];
  f_sqr(f, PP, P);
  f_mul(f, PPP, P, PP);
  f_mul(f, Q, p->x, PP);
  f_sqr(f, X3, R);
  f_sub(f, X3, X3, PPP);
  f_sub(f, X3, X3, Q);
  f_sub(f, X3, X3, Q);
  f_sub(f, t, Q, X3);
  f_mul(f, Y3, R, t);
  f_mul(f, t, p->y, PPP);
  f_sub(f, Y3, Y3, t);
  f_mul(f, r->zz, p->zz, PP);
  f_mul(f, r->zzz, p->zzz, PPP);
  memcpy(r->x, X3, 32);
  memcpy(r->y, Y3, 32);
}

/* add-2008-s: XYZZ + XYZZ (src/ec.cuh:495-546) */
static void xyzz_add(xyzz *r, const xyzz *p, const xyzz *q) {
  if (f_is_zero(p->zz)) {
    *r = *q;
    return;
  }
  if (f_is_zero(q->zz)) {
    *r = *p;
    return;
  }
  const field *f = &FQ;
  u64 U1[4], U2[4], S1[4], S2[4], P[4], R[4];
  f_mul(f, U1, p->x, q->zz);
  f_mul(f, U2, q->x, p->zz);
  f_mul(f, S1, p->y, q->zzz);
  f_mul(f, S2, q->y, p->zzz);
  f_sub(f, P, U2, U1);
  f_sub(f, R, S2, S1);
  if (f_is_zero(P) && f_is_zero(R)) {
    xyzz_dbl(r, p);
    return;
  }
  u64 PP[4], PPP[4], Q[4], X3[4], Y3[4], t[4], ZZ3[4], ZZZ3[4];
  f_sqr(f, PP, P);
  f_mul(f, PPP, P, PP);
  f_mul(f, Q, U1, PP);
  f_sqr(f, X3, R);
  f_sub(f, X3, X3, PPP);
  f_sub(f, X3, X3, Q);
  f_sub(f, X3, X3, Q);
  f_sub(f, t, Q, X3);
  f_mul(f, Y3, R, t);
  f_mul(f, t, S1, PPP);
  f_sub(f, Y3, Y3, t);
  f_mul(f, ZZ3, p->zz, q->zz);
  f_mul(f, ZZ3, ZZ3, PP);
  f_mul(f, ZZZ3, p->zzz, q->zzz);
  f_mul(f, ZZZ3, ZZZ3, PPP);
  memcpy(r->x, X3, 32);
  memcpy(r->y, Y3, 32);
  memcpy(r->zz, ZZ3, 32);
  memcpy(r->zzz, ZZZ3, 32);
}

/* XYZZ -> Jacobian with Z = ZZ*ZZZ (src/ec.cuh:255-263) */
static void xyzz_to_jac(jac *r, const xyzz *p) {
  if (f_is_zero(p->zz)) {
    jac_set_inf(r);
    return;
  }
  const field *f = &FQ;
  u64 z[4], t[4];
  f_mul(f, z, p->zz, p->zzz);
  f_mul(f, t, p->x, p->zzz);
  f_mul(f, r->x, t, z);
  f_mul(f, t, p->y, p->zz);
  u64 z2[4];
  f_sqr(f, z2, z);
  f_mul(f, r->y, t, z2);
  memcpy(r->z, z, 32);
}

static void jac_from_aff(jac *r, const aff *a) {
  memcpy(r->x, a->x, 32);
  memcpy(r->y, a->y, 32);
  memcpy(r->z, FQ.one, 32);
}

/* Jacobian -> standard-form affine; returns 1 for infinity. */
static int jac_normalize(const jac *p, uint32_t out_std[16]) {
  memset(out_std, 0, 64);
  if (f_is_zero(p->z))
    return 1;
  const field *f = &FQ;
  u64 zi[4], zi2[4], zi3[4], x[4], y[4];
  f_inv(f, zi, p->z);
  f_sqr(f, zi2, zi);
  f_mul(f, zi3, zi2, zi);
  f_mul(f, x, p->x, zi2);
  f_mul(f, y, p->y, zi3);
  f_from_mont(f, x, x);
  f_from_mont(f, y, y);
  store8(out_std, x);
  store8(out_std + 8, y);
  return 0;
}

/* Double-and-add from the most significant bit (src/ec.cuh:733-819). */
static void jac_mul(jac *r, const jac *p, const u64 k[4]) {
  jac acc;
  jac_set_inf(&acc);
  for (int i = 255; i >= 0; i--) {
    jac_dbl(&acc, &acc);
    if ((k[i / 64] >> (i % 64)) & 1)
      jac_add(&acc, &acc, p);
  }
  *r = acc;
}

static void load_aff(aff *a, const uint32_t *w) {
  load8(a->x, w);
  load8(a->y, w + 8);
}

static void load_jac(jac *a, const uint32_t *w) {
  load8(a->x, w);
  load8(a->y, w + 8);
  load8(a->z, w + 16);
}

/* ------------------------------------------------------------------------ */
/* Exported field helpers                                                     */
/* ------------------------------------------------------------------------ */
void orc_fq_mul(const uint32_t a[8], const uint32_t b[8], uint32_t out[8]) {
  INIT();
  u64 x[4], y[4], z[4];
  load8(x, a);
  load8(y, b);
  f_mul(&FQ, z, x, y);
  store8(out, z);
}

void orc_fq_to_mont(const uint32_t a[8], uint32_t out[8]) {
  INIT();
  u64 x[4];
  load8(x, a);
  f_to_mont(&FQ, x, x);
  store8(out, x);
}

void orc_fq_from_mont(const uint32_t a[8], uint32_t out[8]) {
  INIT();
  u64 x[4];
  load8(x, a);
  f_from_mont(&FQ, x, x);
  store8(out, x);
}

void orc_fr_to_mont(const uint32_t a[8], uint32_t out[8]) {
  INIT();
  u64 x[4];
  load8(x, a);
  f_to_mont(&FR, x, x);
  store8(out, x);
}

void orc_fr_from_mont(const uint32_t a[8], uint32_t out[8]) {
  INIT();
  u64 x[4];
  load8(x, a);
  f_from_mont(&FR, x, x);
  store8(out, x);
}

void orc_fr_to_mont_batch(const uint32_t *a, uint32_t *out, size_t n) {
  INIT();
  for (size_t i = 0; i < n; i++)
    orc_fr_to_mont(a + 8 * i, out + 8 * i);
}

/* ------------------------------------------------------------------------ */
/* Fixed-base multiples of G = (1, 2)                                         */
/* ------------------------------------------------------------------------ */
static aff G_POW2[256]; /* 2^j * G, Montgomery affine */
static pthread_once_t gtab_once = PTHREAD_ONCE_INIT;

static void gtab_init(void) {
  INIT();
  u64 one_std[4] = {1, 0, 0, 0}, two_std[4] = {2, 0, 0, 0};
  jac g;
  f_to_mont(&FQ, g.x, one_std);
  f_to_mont(&FQ, g.y, two_std);
  memcpy(g.z, FQ.one, 32);
  for (int j = 0; j < 256; j++) {
    uint32_t w[16];
    jac_normalize(&g, w);
    u64 x[4], y[4];
    load8(x, w);
    load8(y, w + 8);
    f_to_mont(&FQ, G_POW2[j].x, x);
    f_to_mont(&FQ, G_POW2[j].y, y);
    jac_dbl(&g, &g);
  }
}

static void mul_gen(xyzz *r, const u64 k[4]) {
  xyzz acc;
  xyzz_set_inf(&acc);
  for (int j = 0; j < 256; j++)
    if ((k[j / 64] >> (j % 64)) & 1)
      xyzz_madd(&acc, &acc, &G_POW2[j]);
  *r = acc;
}

typedef struct {
  const uint32_t *k;
  uint32_t *out;
  size_t begin, end;
  int bad;
} gen_job;

static void *gen_worker(void *arg) {
  gen_job *job = (gen_job *)arg;
  for (size_t i = job->begin; i < job->end; i++) {
    u64 k[4];
    load8(k, job->k + 8 * i);
    if (f_is_zero(k) || geq(k, FR.m)) {
      job->bad = 1;
      continue;
    }
    xyzz p;
    mul_gen(&p, k);
    jac j;
    xyzz_to_jac(&j, &p);
    uint32_t w[16];
    jac_normalize(&j, w);
    u64 x[4], y[4];
    load8(x, w);
    load8(y, w + 8);
    f_to_mont(&FQ, x, x);
    f_to_mont(&FQ, y, y);
    store8(job->out + 16 * i, x);
    store8(job->out + 16 * i + 8, y);
  }
  return NULL;
}

static int default_threads(int threads) {
  if (threads > 0)
    return threads;
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

int orc_gen_bases(const uint32_t *k_std, size_t n, uint32_t *bases_mont, int threads) {
  pthread_once(&gtab_once, gtab_init);
  threads = default_threads(threads);
  if ((size_t)threads > n)
    threads = n ? (int)n : 1;
  gen_job *jobs = calloc(threads, sizeof *jobs);
  pthread_t *tids = calloc(threads, sizeof *tids);
  for (int t = 0; t < threads; t++) {
    jobs[t].k = k_std;
    jobs[t].out = bases_mont;
    jobs[t].begin = n * t / threads;
    jobs[t].end = n * (t + 1) / threads;
    pthread_create(&tids[t], NULL, gen_worker, &jobs[t]);
  }
  int bad = 0;
  for (int t = 0; t < threads; t++) {
    pthread_join(tids[t], NULL);
    bad |= jobs[t].bad;
  }
  free(jobs);
  free(tids);
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Reference-facing reductions                                                */
/* ------------------------------------------------------------------------ */
int orc_jacobian_normalize(const uint32_t jac_mont[24], uint32_t out_std[16]) {
  INIT();
  jac p;
  load_jac(&p, jac_mont);
  return jac_normalize(&p, out_std);
}

/* The caller-side final reduction of the 254 per-bit results
 * (src/bellman-cuda.h:496-505): sum = R[n-1]; sum = 2*sum + R[i] downwards. */
int orc_horner(const uint32_t *results_jac_mont, size_t count, uint32_t out_std[16]) {
  INIT();
  jac sum;
  jac_set_inf(&sum);
  for (size_t i = 0; i < count; i++) {
    size_t index = count - i - 1;
    jac b;
    load_jac(&b, results_jac_mont + 24 * index);
    if (i == 0) {
      sum = b;
    } else {
      jac_dbl(&sum, &sum);
      jac_add(&sum, &sum, &b);
    }
  }
  return jac_normalize(&sum, out_std);
}

int orc_msm_naive(const uint32_t *bases_mont, const uint32_t *scalars_mont, size_t n, uint32_t out_std[16]) {
  INIT();
  jac sum;
  jac_set_inf(&sum);
  for (size_t i = 0; i < n; i++) {
    u64 s[4];
    load8(s, scalars_mont + 8 * i);
    f_from_mont(&FR, s, s);
    aff a;
    load_aff(&a, bases_mont + 16 * i);
    jac p, t;
    jac_from_aff(&p, &a);
    jac_mul(&t, &p, s);
    jac_add(&sum, &sum, &t);
  }
  return jac_normalize(&sum, out_std);
}

/* Checksum oracle of the reference MSM test (tests/msm_test.cu:27-32, 107-114). */
int orc_msm_checksum(const uint32_t *k_std, const uint32_t *scalars_mont, size_t n, uint32_t out_std[16]) {
  INIT();
  pthread_once(&gtab_once, gtab_init);
  u64 acc[4] = {0, 0, 0, 0};
  for (size_t i = 0; i < n; i++) {
    u64 k[4], s[4], km[4], prod[4];
    load8(k, k_std + 8 * i);
    load8(s, scalars_mont + 8 * i);
    f_to_mont(&FR, km, k);
    f_mul(&FR, prod, km, s); /* Montgomery form of k*s */
    f_add(&FR, acc, acc, prod);
  }
  f_from_mont(&FR, acc, acc);
  xyzz p;
  mul_gen(&p, acc);
  jac j;
  xyzz_to_jac(&j, &p);
  return jac_normalize(&j, out_std);
}

int orc_affine_is_on_curve(const uint32_t aff_mont[16]) {
  INIT();
  aff a;
  load_aff(&a, aff_mont);
  u64 y2[4], x3[4], b[4], three[4] = {3, 0, 0, 0};
  f_sqr(&FQ, y2, a.y);
  f_sqr(&FQ, x3, a.x);
  f_mul(&FQ, x3, x3, a.x);
  f_to_mont(&FQ, b, three);
  f_add(&FQ, x3, x3, b);
  return f_eq(y2, x3);
}

static void aff_std_to_jac(jac *j, const uint32_t w[16]) {
  u64 x[4], y[4];
  load8(x, w);
  load8(y, w + 8);
  f_to_mont(&FQ, j->x, x);
  f_to_mont(&FQ, j->y, y);
  memcpy(j->z, FQ.one, 32);
}

int orc_affine_mul(const uint32_t aff_std[16], const uint32_t k_std[8], uint32_t out_std[16]) {
  INIT();
  jac p, r;
  aff_std_to_jac(&p, aff_std);
  u64 k[4];
  load8(k, k_std);
  jac_mul(&r, &p, k);
  return jac_normalize(&r, out_std);
}

int orc_affine_add(const uint32_t a_std[16], int a_inf, const uint32_t b_std[16], int b_inf, uint32_t out_std[16]) {
  INIT();
  jac p, q, r;
  if (a_inf)
    jac_set_inf(&p);
  else
    aff_std_to_jac(&p, a_std);
  if (b_inf)
    jac_set_inf(&q);
  else
    aff_std_to_jac(&q, b_std);
  jac_add(&r, &p, &q);
  return jac_normalize(&r, out_std);
}

/* ------------------------------------------------------------------------ */
/* Multithreaded host Pippenger (the CPU baseline).                           */
/* Signed c-bit digits of min(s, r - s) as in the reference digit kernel      */
/* (src/msm_kernels.cu:36-83), XYZZ buckets, running-sum bucket reduction.    */
/* Tasks are (window, slice of points); a slice's window sum is combined on   */
/* the calling thread.                                                         */
/* ------------------------------------------------------------------------ */
typedef struct {
  const uint32_t *bases;
  const int32_t *digits; /* n x windows, signed */
  size_t n;
  unsigned c, windows, slices;
  xyzz *partials; /* windows x slices */
  size_t next;    /* task counter (protected by lock) */
  pthread_mutex_t lock;
} pip_ctx;

static void *pip_worker(void *arg) {
  pip_ctx *ctx = (pip_ctx *)arg;
  const size_t nb = (size_t)1 << (ctx->c - 1);
  xyzz *buckets = malloc(sizeof(xyzz) * nb);
  for (;;) {
    pthread_mutex_lock(&ctx->lock);
    size_t task = ctx->next++;
    pthread_mutex_unlock(&ctx->lock);
    if (task >= (size_t)ctx->windows * ctx->slices)
      break;
    unsigned w = task / ctx->slices, s = task % ctx->slices;
    size_t begin = ctx->n * s / ctx->slices, end = ctx->n * (s + 1) / ctx->slices;
    for (size_t b = 0; b < nb; b++)
      xyzz_set_inf(&buckets[b]);
    for (size_t i = begin; i < end; i++) {
      int32_t d = ctx->digits[i * ctx->windows + w];
      if (d == 0)
        continue;
      aff a;
      load_aff(&a, ctx->bases + 16 * i);
      if (d < 0) {
        f_neg(&FQ, a.y, a.y);
        d = -d;
      }
      xyzz_madd(&buckets[d - 1], &buckets[d - 1], &a);
    }
    xyzz run, acc;
    xyzz_set_inf(&run);
    xyzz_set_inf(&acc);
    for (size_t b = nb; b-- > 0;) {
      xyzz_add(&run, &run, &buckets[b]);
      xyzz_add(&acc, &acc, &run);
    }
    ctx->partials[task] = acc;
  }
  free(buckets);
  return NULL;
}

static unsigned pip_window_bits(size_t n) {
  unsigned lg = 0;
  while (((size_t)1 << (lg + 1)) <= n)
    lg++;
  if (lg < 4)
    return 3;
  unsigned c = lg - 3;
  if (c > 16)
    c = 16;
  return c;
}

int orc_msm_pippenger(const uint32_t *bases_mont, const uint32_t *scalars_mont, size_t n, int threads, uint32_t out_std[16]) {
  INIT();
  threads = default_threads(threads);
  const unsigned c = pip_window_bits(n);
  const unsigned windows = (254 + c - 1) / c;
  int32_t *digits = malloc(sizeof(int32_t) * (n ? n : 1) * windows);
  for (size_t i = 0; i < n; i++) {
    u64 s[4], neg[4];
    load8(s, scalars_mont + 8 * i);
    f_from_mont(&FR, s, s);
    sub4(neg, FR.m, s);
    int flip = 0;
    if (!geq(neg, s)) { /* r - s < s: digits of r - s, every sign flipped */
      memcpy(s, neg, 32);
      flip = 1;
    }
    unsigned carry = 0;
    for (unsigned w = 0; w < windows; w++) {
      unsigned bit = w * c;
      unsigned limb = bit / 64, off = bit % 64;
      u64 v = limb < 4 ? s[limb] >> off : 0;
      if (off + c > 64 && limb + 1 < 4)
        v |= s[limb + 1] << (64 - off);
      unsigned raw = (unsigned)(v & (((u64)1 << c) - 1)) + carry;
      int32_t d;
      if (raw > (1u << (c - 1))) {
        d = (int32_t)raw - (int32_t)(1u << c);
        carry = 1;
      } else {
        d = (int32_t)raw;
        carry = 0;
      }
      digits[i * windows + w] = flip ? -d : d;
    }
  }
  unsigned slices = 1;
  while (windows * slices < (unsigned)threads * 2 && ((size_t)slices << 1) <= (n ? n : 1))
    slices <<= 1;
  pip_ctx ctx;
  ctx.bases = bases_mont;
  ctx.digits = digits;
  ctx.n = n;
  ctx.c = c;
  ctx.windows = windows;
  ctx.slices = slices;
  ctx.partials = malloc(sizeof(xyzz) * windows * slices);
  ctx.next = 0;
  pthread_mutex_init(&ctx.lock, NULL);
  pthread_t *tids = calloc(threads, sizeof *tids);
  for (int t = 0; t < threads; t++)
    pthread_create(&tids[t], NULL, pip_worker, &ctx);
  for (int t = 0; t < threads; t++)
    pthread_join(tids[t], NULL);
  xyzz total;
  xyzz_set_inf(&total);
  for (unsigned w = windows; w-- > 0;) {
    for (unsigned k = 0; k < c; k++)
      xyzz_dbl(&total, &total);
    for (unsigned s = 0; s < slices; s++)
      xyzz_add(&total, &total, &ctx.partials[w * slices + s]);
  }
  pthread_mutex_destroy(&ctx.lock);
  free(ctx.partials);
  free(tids);
  free(digits);
  jac j;
  xyzz_to_jac(&j, &total);
  return jac_normalize(&j, out_std);
}
