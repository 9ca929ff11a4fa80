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
