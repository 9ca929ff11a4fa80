/*
 * CPU oracle for the BLS12-446 MSM path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference host arithmetic; every function names
 * the reference file:line it follows (paths inside pdroalves/gpu_msm).  Only
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py use
 * it, and only as the checker.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* Constants of src/fp.cu:15-33 (p, R^2 mod p, p' = -p^-1 mod 2^64). */
static const orc_fp P = {{0x311c0026aab0aaabULL, 0x56ee4528c573b5ccULL,
                          0x824e6dc3e23acdeeULL, 0x0f75a64bbac71602ULL,
                          0x0095a4b78a02fe32ULL, 0x200fc34965aad640ULL,
                          0x3cdee0fb28c5e535ULL}};
static const orc_fp R2 = {{0x2AFF01DDDC752B45ULL, 0x92C772A7421CCF5BULL,
                           0x140EEF29C347DAD6ULL, 0xF5A1400C22EA595EULL,
                           0x99D91C9FEC145218ULL, 0x3BB6537F90143D4BULL,
                           0x3627854C9BE7974FULL}};
static const uint64_t P_PRIME = 0xcd63fd900035fffdULL;

/* ------------------------------------------------------------------------ */
/* Fp: src/fp.cu                                                            */
/* ------------------------------------------------------------------------ */

static int fp_cmp(const orc_fp *a, const orc_fp *b) { /* fp.cu:92 */
  for (int i = ORC_LIMBS - 1; i >= 0; i--) {
    if (a->limb[i] > b->limb[i]) return 1;
    if (a->limb[i] < b->limb[i]) return -1;
  }
  return 0;
}

static bool fp_is_zero(const orc_fp *a) { /* fp.cu:100 */
  uint64_t acc = 0;
  for (int i = 0; i < ORC_LIMBS; i++) acc |= a->limb[i];
  return acc == 0;
}

static void fp_set_u64(orc_fp *a, uint64_t v) {
  memset(a, 0, sizeof(*a));
  a->limb[0] = v;
}

static uint64_t fp_add_raw(orc_fp *c, const orc_fp *a, const orc_fp *b) { /* fp.cu:148 */
  u128 carry = 0;
  for (int i = 0; i < ORC_LIMBS; i++) {
    carry += (u128)a->limb[i] + b->limb[i];
    c->limb[i] = (uint64_t)carry;
    carry >>= 64;
  }
  return (uint64_t)carry;
}

static uint64_t fp_sub_raw(orc_fp *c, const orc_fp *a, const orc_fp *b) { /* fp.cu:164 */
  uint64_t borrow = 0;
  for (int i = 0; i < ORC_LIMBS; i++) {
    u128 d = (u128)a->limb[i] - b->limb[i] - borrow;
    c->limb[i] = (uint64_t)d;
    borrow = (uint64_t)(d >> 64) ? 1 : 0;
  }
  return borrow;
}

/* fp.cu:181 -- one conditional subtraction of p */
void orc_fp_add(orc_fp *c, const orc_fp *a, const orc_fp *b) {
  orc_fp s;
  uint64_t carry = fp_add_raw(&s, a, b);
  if (carry || fp_cmp(&s, &P) >= 0) fp_sub_raw(&s, &s, &P);
  *c = s;
}

/* fp.cu:197 -- one conditional addition of p */
void orc_fp_sub(orc_fp *c, const orc_fp *a, const orc_fp *b) {
  orc_fp d;
  uint64_t borrow = fp_sub_raw(&d, a, b);
  if (borrow) fp_add_raw(&d, &d, &P);
  *c = d;
}

/* fp.cu:436 */
void orc_fp_neg(orc_fp *c, const orc_fp *a) {
  if (fp_is_zero(a)) {
    memset(c, 0, sizeof(*c));
  } else {
    orc_fp t = *a;
    orc_fp_sub(c, &P, &t);
  }
}

/* fp.cu:249 schoolbook 7x7 product into 14 words */
static void fp_mul_raw(uint64_t t[2 * ORC_LIMBS], const orc_fp *a, const orc_fp *b) {
  memset(t, 0, 2 * ORC_LIMBS * sizeof(uint64_t));
  for (int i = 0; i < ORC_LIMBS; i++) {
    u128 carry = 0;
    for (int j = 0; j < ORC_LIMBS; j++) {
      carry += (u128)a->limb[i] * b->limb[j] + t[i + j];
      t[i + j] = (uint64_t)carry;
      carry >>= 64;
    }
    t[i + ORC_LIMBS] = (uint64_t)carry;
  }
}

/* fp.cu:306 SOS Montgomery reduction, one final conditional subtraction */
static void fp_mont_reduce(orc_fp *c, const uint64_t in[2 * ORC_LIMBS]) {
  uint64_t t[2 * ORC_LIMBS + 1];
  memcpy(t, in, 2 * ORC_LIMBS * sizeof(uint64_t));
  t[2 * ORC_LIMBS] = 0;
  for (int i = 0; i < ORC_LIMBS; i++) {
    uint64_t m = t[i] * P_PRIME;
    u128 carry = 0;
    for (int j = 0; j < ORC_LIMBS; j++) {
      carry += (u128)m * P.limb[j] + t[i + j];
      t[i + j] = (uint64_t)carry;
      carry >>= 64;
    }
    for (int k = i + ORC_LIMBS; carry != 0 && k <= 2 * ORC_LIMBS; k++) {
      carry += t[k];
      t[k] = (uint64_t)carry;
      carry >>= 64;
    }
  }
  for (int i = 0; i < ORC_LIMBS; i++) c->limb[i] = t[i + ORC_LIMBS];
  if (t[2 * ORC_LIMBS] != 0 || fp_cmp(c, &P) >= 0) fp_sub_raw(c, c, &P);
}

/* fp.cu:370 */
void orc_fp_mont_mul(orc_fp *c, const orc_fp *a, const orc_fp *b) {
  uint64_t t[2 * ORC_LIMBS];
  fp_mul_raw(t, a, b);
  fp_mont_reduce(c, t);
}

/* fp.cu:378 */
void orc_fp_to_mont(orc_fp *c, const orc_fp *a) { orc_fp_mont_mul(c, a, &R2); }

/* fp.cu:389 */
void orc_fp_from_mont(orc_fp *c, const orc_fp *a) {
  uint64_t t[2 * ORC_LIMBS] = {0};
  for (int i = 0; i < ORC_LIMBS; i++) t[i] = a->limb[i];
  fp_mont_reduce(c, t);
}

/* fp.cu:424 normal-form product via Montgomery */
void orc_fp_mul(orc_fp *c, const orc_fp *a, const orc_fp *b) {
  orc_fp am, bm, cm;
  orc_fp_to_mont(&am, a);
  orc_fp_to_mont(&bm, b);
  orc_fp_mont_mul(&cm, &am, &bm);
  orc_fp_from_mont(c, &cm);
}

/* fp.cu:448 square-and-multiply, base in normal form, result normal form */
static void fp_pow_internal(orc_fp *res, const orc_fp *base, const uint64_t *e, int e_limbs) {
  orc_fp bm, acc, one;
  orc_fp_to_mont(&bm, base);
  fp_set_u64(&one, 1);
  orc_fp_to_mont(&acc, &one);
  int top = e_limbs - 1;
  while (top >= 0 && e[top] == 0) top--;
  for (int l = top; l >= 0; l--) {
    int start = 63;
    if (l == top) {
      while (start >= 0 && ((e[l] >> start) & 1) == 0) start--;
    }
    for (int bit = start; bit >= 0; bit--) {
      orc_fp_mont_mul(&acc, &acc, &acc);
      if ((e[l] >> bit) & 1) orc_fp_mont_mul(&acc, &acc, &bm);
    }
  }
  orc_fp_from_mont(res, &acc);
}

void orc_fp_pow(orc_fp *c, const orc_fp *a, const uint64_t *e, int e_limbs) { /* fp.cu:513 */
  if (e_limbs > ORC_LIMBS) e_limbs = ORC_LIMBS;
  fp_pow_internal(c, a, e, e_limbs);
}

/* fp.cu:522 Fermat inverse of a normal-form value; 0 -> 0 */
void orc_fp_inv(orc_fp *c, const orc_fp *a) {
  if (fp_is_zero(a)) {
    memset(c, 0, sizeof(*c));
    return;
  }
  orc_fp e = P;
  e.limb[0] -= 2; /* p is odd and > 2: no borrow */
  fp_pow_internal(c, a, e.limb, ORC_LIMBS);
}

/* fp.cu:545 Montgomery-form inverse; 0 -> 0 */
void orc_fp_mont_inv(orc_fp *c, const orc_fp *a) {
  if (fp_is_zero(a)) {
    memset(c, 0, sizeof(*c));
    return;
  }
  orc_fp an, rn;
  orc_fp_from_mont(&an, a);
  orc_fp_inv(&rn, &an);
  orc_fp_to_mont(c, &rn);
}

void orc_fp_mont_mul_batch(orc_fp *c, const orc_fp *a, const orc_fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp_mont_mul(&c[i], &a[i], &b[i]);
}
void orc_fp_mul_batch(orc_fp *c, const orc_fp *a, const orc_fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp_mul(&c[i], &a[i], &b[i]);
}
void orc_fp_to_mont_batch(orc_fp *c, const orc_fp *a, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp_to_mont(&c[i], &a[i]);
}
void orc_fp_from_mont_batch(orc_fp *c, const orc_fp *a, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp_from_mont(&c[i], &a[i]);
}

/* ------------------------------------------------------------------------ */
/* Fp2 = Fp[i]/(i^2+1): src/fp2.cu                                          */
/* ------------------------------------------------------------------------ */

static int fp2_cmp(const orc_fp2 *a, const orc_fp2 *b) { /* fp2.cu:4 */
  int c = fp_cmp(&a->c0, &b->c0);
  return c != 0 ? c : fp_cmp(&a->c1, &b->c1);
}
static bool fp2_is_zero(const orc_fp2 *a) { return fp_is_zero(&a->c0) && fp_is_zero(&a->c1); }

void orc_fp2_add(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b) { /* fp2.cu:41 */
  orc_fp_add(&c->c0, &a->c0, &b->c0);
  orc_fp_add(&c->c1, &a->c1, &b->c1);
}
void orc_fp2_sub(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b) { /* fp2.cu:48 */
  orc_fp_sub(&c->c0, &a->c0, &b->c0);
  orc_fp_sub(&c->c1, &a->c1, &b->c1);
}
static void fp2_neg(orc_fp2 *c, const orc_fp2 *a) { /* fp2.cu:143 */
  orc_fp_neg(&c->c0, &a->c0);
  orc_fp_neg(&c->c1, &a->c1);
}

/* fp2.cu:88-112 Karatsuba: t0=a0b0, t1=a1b1, t2=(a0+a1)(b0+b1) */
void orc_fp2_mont_mul(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b) {
  orc_fp t0, t1, t2, t3;
  orc_fp_mont_mul(&t0, &a->c0, &b->c0);
  orc_fp_mont_mul(&t1, &a->c1, &b->c1);
  orc_fp_add(&t2, &a->c0, &a->c1);
  orc_fp_add(&t3, &b->c0, &b->c1);
  orc_fp_mont_mul(&t2, &t2, &t3);
  orc_fp_sub(&c->c0, &t0, &t1);
  orc_fp_sub(&c->c1, &t2, &t0);
  orc_fp_sub(&c->c1, &c->c1, &t1);
}

/* fp2.cu:58-82 normal-form product */
void orc_fp2_mul(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b) {
  orc_fp t0, t1, t2, t3;
  orc_fp_mul(&t0, &a->c0, &b->c0);
  orc_fp_mul(&t1, &a->c1, &b->c1);
  orc_fp_add(&t2, &a->c0, &a->c1);
  orc_fp_add(&t3, &b->c0, &b->c1);
  orc_fp_mul(&t2, &t2, &t3);
  orc_fp_sub(&c->c0, &t0, &t1);
  orc_fp_sub(&c->c1, &t2, &t0);
  orc_fp_sub(&c->c1, &c->c1, &t1);
}

/* fp2.cu:232 inverse via the norm a0^2 + a1^2 */
void orc_fp2_mont_inv(orc_fp2 *c, const orc_fp2 *a) {
  if (fp2_is_zero(a)) {
    memset(c, 0, sizeof(*c));
    return;
  }
  orc_fp t0, t1, norm, ninv, na1;
  orc_fp_mont_mul(&t0, &a->c0, &a->c0);
  orc_fp_mont_mul(&t1, &a->c1, &a->c1);
  orc_fp_add(&norm, &t0, &t1);
  orc_fp_mont_inv(&ninv, &norm);
  orc_fp_mont_mul(&c->c0, &a->c0, &ninv);
  orc_fp_neg(&na1, &a->c1);
  orc_fp_mont_mul(&c->c1, &na1, &ninv);
}

void orc_fp2_mont_mul_batch(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp2_mont_mul(&c[i], &a[i], &b[i]);
}
void orc_fp2_mul_batch(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) orc_fp2_mul(&c[i], &a[i], &b[i]);
}

/* ------------------------------------------------------------------------ */
/* Field-generic glue for the curve templates                               */
/* ------------------------------------------------------------------------ */

static void fp_const(orc_fp *c, uint64_t k) { /* k in Montgomery form */
  orc_fp t;
  fp_set_u64(&t, k);
  orc_fp_to_mont(c, &t);
}
static void fp2_const(orc_fp2 *c, uint64_t k) {
  fp_const(&c->c0, k);
  memset(&c->c1, 0, sizeof(c->c1));
}
static bool fp_eq(const orc_fp *a, const orc_fp *b) { return fp_cmp(a, b) == 0; }
static bool fp2_eq(const orc_fp2 *a, const orc_fp2 *b) { return fp2_cmp(a, b) == 0; }

/* G1 instantiation */
#define F orc_fp
#define F_ADD orc_fp_add
#define F_SUB orc_fp_sub
#define F_NEG orc_fp_neg
#define F_MUL orc_fp_mont_mul
#define F_INV orc_fp_mont_inv
#define F_ISZERO fp_is_zero
#define F_EQ fp_eq
#define F_CONST fp_const
#define AFF orc_g1
#define PRJ orc_g1p
#define PFX(name) orc_g1_##name
#define PPFX(name) orc_g1p_##name
#define SPFX(name) g1_##name
#include "oracle_curve.inc"
#undef F
#undef F_ADD
#undef F_SUB
#undef F_NEG
#undef F_MUL
#undef F_INV
#undef F_ISZERO
#undef F_EQ
#undef F_CONST
#undef AFF
#undef PRJ
#undef PFX
#undef PPFX
#undef SPFX

/* G2 instantiation */
#define F orc_fp2
#define F_ADD orc_fp2_add
#define F_SUB orc_fp2_sub
#define F_NEG fp2_neg
#define F_MUL orc_fp2_mont_mul
#define F_INV orc_fp2_mont_inv
#define F_ISZERO fp2_is_zero
#define F_EQ fp2_eq
#define F_CONST fp2_const
#define AFF orc_g2
#define PRJ orc_g2p
#define PFX(name) orc_g2_##name
#define PPFX(name) orc_g2p_##name
#define SPFX(name) g2_##name
#include "oracle_curve.inc"

/* ------------------------------------------------------------------------ */
/* Generators (standard form), src/curve.cu:786-814                         */
/* ------------------------------------------------------------------------ */

void orc_g1_generator(orc_g1 *g) {
  static const orc_g1 G = {
      {{0x3bf9166c8236f4faULL, 0x8bc02b7cbe6a9e8dULL, 0x11c1e56b3e4bc80bULL,
        0x6b20d782901a6f62ULL, 0x2ce8c34265bf3841ULL, 0x11b73d3d76ae9851ULL,
        0x326ed6bd777fc6a3ULL}},
      {{0xfe6f792612016b30ULL, 0x22db0ce6034a9db9ULL, 0xb9093f32002756daULL,
        0x39d7f424b6660204ULL, 0xf843c947aa57f571ULL, 0xd6d62d244e413636ULL,
        0x1a7caf4a4d3887a6ULL}},
      false};
  *g = G;
}

void orc_g2_generator(orc_g2 *g) {
  static const orc_g2 G = {
      {{{0x0e529ee4dce9991dULL, 0xd6ebaf149094f1ccULL, 0x043c6bf16312d638ULL,
         0x062b61439640e885ULL, 0x18dad8ed784dd225ULL, 0xa57c0038441f7d15ULL,
         0x21f8d4a76f74541aULL}},
       {{0xcaf5185423a7d23aULL, 0x7cef6acb145b6413ULL, 0x2879dd439b019b8bULL,
         0x71449cdeca4f0007ULL, 0xdebaf4a2c5534527ULL, 0xa1b4e791d1b86560ULL,
         0x1e0f563c601bb8dcULL}}},
      {{{0x274315837455b919ULL, 0x82039e4221ff3507ULL, 0x00346cebad16a036ULL,
         0x0177bfd6654e681eULL, 0xddff621b5db3f897ULL, 0x0cc61570301497a7ULL,
         0x115ea2305a78f646ULL}},
       {{0x392236e9cf2976c2ULL, 0xd8ab17c84b9f03cdULL, 0x8a8e6755f9d82fd1ULL,
         0x7532834528cd5a64ULL, 0x0b0bcc3fb6f2161cULL, 0x76a2ffcb7d47679dULL,
         0x25ed2192b203c1feULL}}},
      false};
  *g = G;
}

void orc_g1_to_mont(orc_g1 *r, const orc_g1 *p) { /* curve.cu:2333 */
  orc_g1 t = *p;
  if (t.infinity) {
    memset(r, 0, sizeof(*r));
    r->infinity = true;
    return;
  }
  orc_fp_to_mont(&t.x, &p->x);
  orc_fp_to_mont(&t.y, &p->y);
  *r = t;
}
void orc_g1_from_mont(orc_g1 *r, const orc_g1 *p) { /* c_wrapper.cu:261 */
  orc_g1 t = *p;
  if (t.infinity) {
    memset(r, 0, sizeof(*r));
    r->infinity = true;
    return;
  }
  orc_fp_from_mont(&t.x, &p->x);
  orc_fp_from_mont(&t.y, &p->y);
  *r = t;
}
void orc_g2_to_mont(orc_g2 *r, const orc_g2 *p) {
  orc_g2 t = *p;
  if (t.infinity) {
    memset(r, 0, sizeof(*r));
    r->infinity = true;
    return;
  }
  orc_fp_to_mont(&t.x.c0, &p->x.c0);
  orc_fp_to_mont(&t.x.c1, &p->x.c1);
  orc_fp_to_mont(&t.y.c0, &p->y.c0);
  orc_fp_to_mont(&t.y.c1, &p->y.c1);
  *r = t;
}
void orc_g2_from_mont(orc_g2 *r, const orc_g2 *p) { /* c_wrapper.cu:271 */
  orc_g2 t = *p;
  if (t.infinity) {
    memset(r, 0, sizeof(*r));
    r->infinity = true;
    return;
  }
  orc_fp_from_mont(&t.x.c0, &p->x.c0);
  orc_fp_from_mont(&t.x.c1, &p->x.c1);
  orc_fp_from_mont(&t.y.c0, &p->y.c0);
  orc_fp_from_mont(&t.y.c1, &p->y.c1);
  *r = t;
}

/* On-curve checks.  The reference declares b = 4 and b' = 4i
 * (src/curve.cu:280-289) but its generators satisfy y^2 = x^3 + 1 (G1) and
 * y^2 = x^3 + (1 + i) (G2); the checker uses the constants the points
 * actually satisfy. */
bool orc_g1_on_curve(const orc_g1 *p) {
  if (p->infinity) return true;
  orc_fp y2, x2, x3, b, rhs;
  orc_fp_mont_mul(&y2, &p->y, &p->y);
  orc_fp_mont_mul(&x2, &p->x, &p->x);
  orc_fp_mont_mul(&x3, &x2, &p->x);
  fp_const(&b, 1);
  orc_fp_add(&rhs, &x3, &b);
  return fp_eq(&y2, &rhs);
}
bool orc_g2_on_curve(const orc_g2 *p) {
  if (p->infinity) return true;
  orc_fp2 y2, x2, x3, b, rhs;
  orc_fp2_mont_mul(&y2, &p->y, &p->y);
  orc_fp2_mont_mul(&x2, &p->x, &p->x);
  orc_fp2_mont_mul(&x3, &x2, &p->x);
  fp_const(&b.c0, 1);
  fp_const(&b.c1, 1);
  orc_fp2_add(&rhs, &x3, &b);
  return fp2_eq(&y2, &rhs);
}
