// Host-side BLS12-446 arithmetic for the C-ABI helpers that the reference runs
// on the CPU (pdroalves/gpu_msm rust-api/src/c_wrapper.cu:12-59, 261-288):
// Montgomery conversion, affine <-> projective, point-at-infinity helpers.
// 7 x 64-bit limbs, CIOS Montgomery multiplication with 128-bit products.
// All results are canonical (< p), so they agree with the reference's host
// functions bit for bit on canonical inputs.
#pragma once
#include <cstdint>
#include <cstring>

#include "../../include/gpu_msm_b200.h"

namespace gm_host {

typedef unsigned __int128 u128;
constexpr int L = 7;

static const uint64_t P[L] = {0x311c0026aab0aaabULL, 0x56ee4528c573b5ccULL, 0x824e6dc3e23acdeeULL,
                              0x0f75a64bbac71602ULL, 0x0095a4b78a02fe32ULL, 0x200fc34965aad640ULL,
                              0x3cdee0fb28c5e535ULL};
static const uint64_t R2[L] = {0x2AFF01DDDC752B45ULL, 0x92C772A7421CCF5BULL, 0x140EEF29C347DAD6ULL,
                               0xF5A1400C22EA595EULL, 0x99D91C9FEC145218ULL, 0x3BB6537F90143D4BULL,
                               0x3627854C9BE7974FULL};
static const uint64_t PINV64 = 0xcd63fd900035fffdULL;  // -p^-1 mod 2^64

inline bool geq_p(const uint64_t a[L]) {
  for (int i = L - 1; i >= 0; i--) {
    if (a[i] > P[i]) return true;
    if (a[i] < P[i]) return false;
  }
  return true;
}
inline void sub_p(uint64_t a[L]) {
  uint64_t br = 0;
  for (int i = 0; i < L; i++) {
    u128 d = (u128)a[i] - P[i] - br;
    a[i] = (uint64_t)d;
    br = (uint64_t)(d >> 64) ? 1 : 0;
  }
}
inline bool is_zero(const uint64_t a[L]) {
  uint64_t acc = 0;
  for (int i = 0; i < L; i++) acc |= a[i];
  return acc == 0;
}

// c = a*b*R^-1 mod p (CIOS, 64-bit words); canonical for canonical inputs
inline void mont_mul(uint64_t c[L], const uint64_t a[L], const uint64_t b[L]) {
  uint64_t t[L + 2] = {0};
  for (int i = 0; i < L; i++) {
    u128 carry = 0;
    for (int j = 0; j < L; j++) {
      carry += (u128)a[j] * b[i] + t[j];
      t[j] = (uint64_t)carry;
      carry >>= 64;
    }
    carry += t[L];
    t[L] = (uint64_t)carry;
    t[L + 1] = (uint64_t)(carry >> 64);
    const uint64_t m = t[0] * PINV64;
    carry = (u128)m * P[0] + t[0];
    carry >>= 64;
    for (int j = 1; j < L; j++) {
      carry += (u128)m * P[j] + t[j];
      t[j - 1] = (uint64_t)carry;
      carry >>= 64;
    }
    carry += t[L];
    t[L - 1] = (uint64_t)carry;
    t[L] = t[L + 1] + (uint64_t)(carry >> 64);
  }
  uint64_t r[L];
  for (int i = 0; i < L; i++) r[i] = t[i];
  if (t[L] || geq_p(r)) sub_p(r);
  memcpy(c, r, sizeof(r));
}

// c = a^2 R^-1 mod p: the 21 cross products once, doubled, plus the 7
// squares on the diagonal (28 products instead of 49), then the same
// word-by-word Montgomery reduction; canonical for canonical inputs.
inline void mont_sqr(uint64_t c[L], const uint64_t a[L]) {
  uint64_t t[2 * L + 1];
  memset(t, 0, sizeof(t));
  for (int i = 0; i < L - 1; i++) {
    u128 carry = 0;
    for (int j = i + 1; j < L; j++) {
      carry += (u128)a[i] * a[j] + t[i + j];
      t[i + j] = (uint64_t)carry;
      carry >>= 64;
    }
    t[i + L] = (uint64_t)carry;
  }
  uint64_t top = 0;
  for (int k = 0; k < 2 * L; k++) {
    const uint64_t nt = t[k] >> 63;
    t[k] = (t[k] << 1) | top;
    top = nt;
  }
  u128 carry = 0;
  for (int i = 0; i < L; i++) {
    const u128 sq = (u128)a[i] * a[i];
    carry += (u128)t[2 * i] + (uint64_t)sq;
    t[2 * i] = (uint64_t)carry;
    carry >>= 64;
    carry += (u128)t[2 * i + 1] + (uint64_t)(sq >> 64);
    t[2 * i + 1] = (uint64_t)carry;
    carry >>= 64;
  }
  for (int i = 0; i < L; i++) {
    const uint64_t m = t[i] * PINV64;
    u128 cy = 0;
    for (int j = 0; j < L; j++) {
      cy += (u128)m * P[j] + t[i + j];
      t[i + j] = (uint64_t)cy;
      cy >>= 64;
    }
    for (int k = i + L; cy != 0 && k < 2 * L + 1; k++) {
      cy += t[k];
      t[k] = (uint64_t)cy;
      cy >>= 64;
    }
  }
  uint64_t r[L];
  for (int i = 0; i < L; i++) r[i] = t[L + i];
  if (t[2 * L] || geq_p(r)) sub_p(r);
  memcpy(c, r, sizeof(r));
}

inline void add(uint64_t c[L], const uint64_t a[L], const uint64_t b[L]) {
  u128 carry = 0;
  uint64_t r[L];
  for (int i = 0; i < L; i++) {
    carry += (u128)a[i] + b[i];
    r[i] = (uint64_t)carry;
    carry >>= 64;
  }
  if (carry || geq_p(r)) sub_p(r);
  memcpy(c, r, sizeof(r));
}
inline void sub(uint64_t c[L], const uint64_t a[L], const uint64_t b[L]) {
  uint64_t r[L], br = 0;
  for (int i = 0; i < L; i++) {
    u128 d = (u128)a[i] - b[i] - br;
    r[i] = (uint64_t)d;
    br = (uint64_t)(d >> 64) ? 1 : 0;
  }
  if (br) {
    u128 carry = 0;
    for (int i = 0; i < L; i++) {
      carry += (u128)r[i] + P[i];
      r[i] = (uint64_t)carry;
      carry >>= 64;
    }
  }
  memcpy(c, r, sizeof(r));
}
inline void neg(uint64_t c[L], const uint64_t a[L]) {
  if (is_zero(a)) {
    memset(c, 0, sizeof(uint64_t) * L);
    return;
  }
  uint64_t t[L];
  memcpy(t, a, sizeof(t));
  sub(c, P, t);
}
inline void to_mont(uint64_t c[L], const uint64_t a[L]) { mont_mul(c, a, R2); }
inline void from_mont(uint64_t c[L], const uint64_t a[L]) {
  uint64_t one[L] = {1, 0, 0, 0, 0, 0, 0};
  mont_mul(c, a, one);
}
inline void one_mont(uint64_t c[L]) {
  uint64_t one[L] = {1, 0, 0, 0, 0, 0, 0};
  to_mont(c, one);
}
// Montgomery-form inverse by Fermat, a^(p-2); 0 -> 0
inline void mont_inv(uint64_t c[L], const uint64_t a[L]) {
  if (is_zero(a)) {
    memset(c, 0, sizeof(uint64_t) * L);
    return;
  }
  uint64_t e[L];
  memcpy(e, P, sizeof(e));
  e[0] -= 2;
  uint64_t acc[L];
  one_mont(acc);
  for (int i = L - 1; i >= 0; i--)
    for (int b = 63; b >= 0; b--) {
      mont_mul(acc, acc, acc);
      if ((e[i] >> b) & 1) mont_mul(acc, acc, a);
    }
  memcpy(c, acc, sizeof(acc));
}

// Fp2 (i^2 = -1)
inline void fp2_mul(Fp2 &c, const Fp2 &a, const Fp2 &b) {
  uint64_t t0[L], t1[L], s0[L], s1[L], t2[L];
  mont_mul(t0, a.c0.limb, b.c0.limb);
  mont_mul(t1, a.c1.limb, b.c1.limb);
  add(s0, a.c0.limb, a.c1.limb);
  add(s1, b.c0.limb, b.c1.limb);
  mont_mul(t2, s0, s1);
  sub(c.c0.limb, t0, t1);
  sub(c.c1.limb, t2, t0);
  sub(c.c1.limb, c.c1.limb, t1);
}
inline bool fp2_is_zero(const Fp2 &a) { return is_zero(a.c0.limb) && is_zero(a.c1.limb); }
inline void fp2_inv(Fp2 &c, const Fp2 &a) {
  if (fp2_is_zero(a)) {
    memset(&c, 0, sizeof(c));
    return;
  }
  uint64_t t0[L], t1[L], nrm[L], ni[L], na1[L];
  mont_mul(t0, a.c0.limb, a.c0.limb);
  mont_mul(t1, a.c1.limb, a.c1.limb);
  add(nrm, t0, t1);
  mont_inv(ni, nrm);
  Fp2 r;
  mont_mul(r.c0.limb, a.c0.limb, ni);
  neg(na1, a.c1.limb);
  mont_mul(r.c1.limb, na1, ni);
  c = r;
}

}  // namespace gm_host

// ---------------------------------------------------------------------------
// Host XYZZ arithmetic for the window combination of a single MSM (the
// serial tail: ~300 doublings).  A CPU core multiplies 446-bit numbers with
// far lower latency than one GPU thread, so the tail runs here, stream-
// ordered through cudaLaunchHostFunc.  Same EFD formulas as xyzz.cuh:
// dbl-2008-s-1 and add-2008-s for a = 0, all values canonical (< p).
// ---------------------------------------------------------------------------
namespace gm_host {

struct HFp {
  uint64_t v[L];
};
struct HFp2 {
  HFp c0, c1;
};

struct F1 {
  using T = HFp;
  static constexpr int WORDS = L;
  static void zero(T &a) { memset(a.v, 0, sizeof(a.v)); }
  static bool is_zero(const T &a) { return gm_host::is_zero(a.v); }
  static void add(T &c, const T &a, const T &b) { gm_host::add(c.v, a.v, b.v); }
  static void sub(T &c, const T &a, const T &b) { gm_host::sub(c.v, a.v, b.v); }
  static void mul(T &c, const T &a, const T &b) { gm_host::mont_mul(c.v, a.v, b.v); }
  static void sqr(T &c, const T &a) { gm_host::mont_sqr(c.v, a.v); }
};

struct F2 {
  using T = HFp2;
  static constexpr int WORDS = 2 * L;
  static void zero(T &a) { memset(&a, 0, sizeof(a)); }
  static bool is_zero(const T &a) { return gm_host::is_zero(a.c0.v) && gm_host::is_zero(a.c1.v); }
  static void add(T &c, const T &a, const T &b) {
    gm_host::add(c.c0.v, a.c0.v, b.c0.v);
    gm_host::add(c.c1.v, a.c1.v, b.c1.v);
  }
  static void sub(T &c, const T &a, const T &b) {
    gm_host::sub(c.c0.v, a.c0.v, b.c0.v);
    gm_host::sub(c.c1.v, a.c1.v, b.c1.v);
  }
  static void mul(T &c, const T &a, const T &b) {
    uint64_t t0[L], t1[L], s0[L], s1[L], t2[L];
    mont_mul(t0, a.c0.v, b.c0.v);
    mont_mul(t1, a.c1.v, b.c1.v);
    gm_host::add(s0, a.c0.v, a.c1.v);
    gm_host::add(s1, b.c0.v, b.c1.v);
    mont_mul(t2, s0, s1);
    gm_host::sub(c.c0.v, t0, t1);
    gm_host::sub(c.c1.v, t2, t0);
    gm_host::sub(c.c1.v, c.c1.v, t1);
  }
  // (a0 + a1 i)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 i
  static void sqr(T &c, const T &a) {
    uint64_t s[L], d[L], m[L];
    gm_host::add(s, a.c0.v, a.c1.v);
    gm_host::sub(d, a.c0.v, a.c1.v);
    mont_mul(m, a.c0.v, a.c1.v);
    mont_mul(c.c0.v, s, d);
    gm_host::add(c.c1.v, m, m);
  }
};

template <class F>
struct HXyzz {
  typename F::T X, Y, ZZ, ZZZ;
};

template <class F>
inline bool hx_is_inf(const HXyzz<F> &p) {
  return F::is_zero(p.ZZ);
}

template <class F>
inline void hx_dbl(HXyzz<F> &p) {
  using T = typename F::T;
  if (hx_is_inf(p)) return;
  T U, V, W, S, xx, M, t, X3, Y3;
  F::add(U, p.Y, p.Y);
  F::mul(V, U, U);
  F::mul(W, U, V);
  F::mul(S, p.X, V);
  F::mul(xx, p.X, p.X);
  F::add(M, xx, xx);
  F::add(M, M, xx);
  F::mul(X3, M, M);
  F::add(t, S, S);
  F::sub(X3, X3, t);
  F::sub(t, S, X3);
  F::mul(Y3, M, t);
  F::mul(t, W, p.Y);
  F::sub(Y3, Y3, t);
  F::mul(p.ZZ, V, p.ZZ);
  F::mul(p.ZZZ, W, p.ZZZ);
  p.X = X3;
  p.Y = Y3;
}

template <class F>
inline void hx_add(HXyzz<F> &acc, const HXyzz<F> &q) {
  using T = typename F::T;
  if (hx_is_inf(q)) return;
  if (hx_is_inf(acc)) {
    acc = q;
    return;
  }
  T U1, U2, S1, S2, P, R, PP, PPP, Q, X3, Y3, t;
  F::mul(U1, acc.X, q.ZZ);
  F::mul(U2, q.X, acc.ZZ);
  F::mul(S1, acc.Y, q.ZZZ);
  F::mul(S2, q.Y, acc.ZZZ);
  F::sub(P, U2, U1);
  F::sub(R, S2, S1);
  if (F::is_zero(P)) {
    if (F::is_zero(R)) {
      hx_dbl(acc);
    } else {
      F::zero(acc.X);
      F::zero(acc.Y);
      F::zero(acc.ZZ);
      F::zero(acc.ZZZ);
    }
    return;
  }
  F::mul(PP, P, P);
  F::mul(PPP, P, PP);
  F::mul(Q, U1, PP);
  F::mul(X3, R, R);
  F::sub(X3, X3, PPP);
  F::add(t, Q, Q);
  F::sub(X3, X3, t);
  F::sub(t, Q, X3);
  F::mul(Y3, R, t);
  F::mul(t, S1, PPP);
  F::sub(Y3, Y3, t);
  F::mul(t, acc.ZZ, q.ZZ);
  F::mul(acc.ZZ, t, PP);
  F::mul(t, acc.ZZZ, q.ZZZ);
  F::mul(acc.ZZZ, t, PPP);
  acc.X = X3;
  acc.Y = Y3;
}

// Jacobian coordinates (x = X/Z^2, y = Y/Z^3) for the runs of c doublings
// of the Horner loop: dbl-2009-l for a = 0 costs 2M + 5S against 6M + 3S
// in XYZZ.  XYZZ -> Jacobian without an inversion: Z' = ZZZ,
// X' = X ZZ^2, Y' = Y ZZZ^2 (since ZZZ^2 = ZZ^3); back: ZZ = Z^2, ZZZ = Z^3.
template <class F>
struct HJac {
  typename F::T X, Y, Z;
};

template <class F>
inline void jac_from_xyzz(HJac<F> &j, const HXyzz<F> &p) {
  typename F::T t;
  F::sqr(t, p.ZZ);
  F::mul(j.X, p.X, t);
  F::sqr(t, p.ZZZ);
  F::mul(j.Y, p.Y, t);
  j.Z = p.ZZZ;
}

template <class F>
inline void xyzz_from_jac(HXyzz<F> &p, const HJac<F> &j) {
  p.X = j.X;
  p.Y = j.Y;
  F::sqr(p.ZZ, j.Z);
  F::mul(p.ZZZ, p.ZZ, j.Z);
}

// 2P in place (dbl-2009-l); Y = 0 or Z = 0 gives Z = 0 (infinity)
template <class F>
inline void jac_dbl(HJac<F> &j) {
  using T = typename F::T;
  T A, B, C, D, E, Fv, t;
  F::sqr(A, j.X);
  F::sqr(B, j.Y);
  F::sqr(C, B);
  F::add(t, j.X, B);
  F::sqr(D, t);
  F::sub(D, D, A);
  F::sub(D, D, C);
  F::add(D, D, D);
  F::add(E, A, A);
  F::add(E, E, A);
  F::sqr(Fv, E);
  F::mul(t, j.Y, j.Z);
  F::add(j.Z, t, t);
  F::add(t, D, D);
  F::sub(j.X, Fv, t);
  F::sub(t, D, j.X);
  F::mul(j.Y, E, t);
  F::add(C, C, C);
  F::add(C, C, C);
  F::add(C, C, C);
  F::sub(j.Y, j.Y, C);
}

// Horner with XYZZ doublings only (dbl-2008-s-1): the reference point for
// gm_host_selftest's check of the Jacobian version below.
template <class F>
inline void horner_xyzz(HXyzz<F> &res, const HXyzz<F> *sums, int W, int c) {
  memset(&res, 0, sizeof(res));
  for (int w = W - 1; w >= 0; w--) {
    if (!hx_is_inf(res))
      for (int k = 0; k < c; k++) hx_dbl(res);
    hx_add(res, sums[w]);
  }
}

// result = sum_w 2^(c w) S_w (Horner, MSB first), then to homogeneous
// projective (X*ZZZ, Y*ZZ, ZZ*ZZZ); infinity -> all zero.  `sums` holds W
// device-layout XYZZ points (32-bit limb order == 64-bit limb order on a
// little-endian host); `out` receives 3 coordinates of F::WORDS u64.
template <class F>
inline void horner_to_proj(uint64_t *out, const HXyzz<F> *sums, int W, int c) {
  HXyzz<F> res;
  memset(&res, 0, sizeof(res));
  HJac<F> j;
  for (int w = W - 1; w >= 0; w--) {
    if (!hx_is_inf(res)) {
      jac_from_xyzz(j, res);
      for (int k = 0; k < c; k++) jac_dbl(j);
      xyzz_from_jac(res, j);
    }
    hx_add(res, sums[w]);
  }
  typename F::T X, Y, Z;
  if (hx_is_inf(res)) {
    memset(out, 0, 3 * F::WORDS * sizeof(uint64_t));
    return;
  }
  F::mul(X, res.X, res.ZZZ);
  F::mul(Y, res.Y, res.ZZ);
  F::mul(Z, res.ZZ, res.ZZZ);
  memcpy(out, &X, F::WORDS * 8);
  memcpy(out + F::WORDS, &Y, F::WORDS * 8);
  memcpy(out + 2 * F::WORDS, &Z, F::WORDS * 8);
}

}  // namespace gm_host
