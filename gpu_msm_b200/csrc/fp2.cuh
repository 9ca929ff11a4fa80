// Fp2 = Fp[i]/(i^2 + 1) on sm_100a (pdroalves/gpu_msm include/fp2.h:7,
// non-residue i as in src/fp2.cu:283-294).  Layout {c0, c1} is
// byte-identical to the reference's `Fp2{Fp c0, c1}` (include/fp2.h:10).
//
// Multiplication is 3-mul Karatsuba (the algorithm of src/fp2.cu:88-112):
//   t0 = a0*b0, t1 = a1*b1, t2 = (a0+a1)*(b0+b1); c0 = t0 - t1, c1 = t2 - t0 - t1.
// Squaring uses the complex method: c0 = (a0+a1)(a0-a1), c1 = 2*a0*a1.
// Every result is the canonical element, so outputs match the reference's
// fp2_mont_mul bit for bit.
#pragma once
#include "field.cuh"

namespace gm {

struct fp2_t {
  fp_t c0, c1;
};

struct Fp2 {
  using T = fp2_t;
  static constexpr int LIMBS = 2 * NL;

  GM_DEVI static fp2_t zero() { return fp2_t{Fp::zero(), Fp::zero()}; }
  GM_DEVI static fp2_t one() { return fp2_t{Fp::one(), Fp::zero()}; }
  GM_DEVI static bool is_zero(const fp2_t &a) { return Fp::is_zero(a.c0) && Fp::is_zero(a.c1); }
  GM_DEVI static bool is_zero_raw(const fp2_t &a) { return Fp::is_zero_raw(a.c0) && Fp::is_zero_raw(a.c1); }
  GM_DEVI static bool eq(const fp2_t &a, const fp2_t &b) { return Fp::eq(a.c0, b.c0) && Fp::eq(a.c1, b.c1); }
  GM_DEVI static fp2_t add(const fp2_t &a, const fp2_t &b) { return fp2_t{Fp::add(a.c0, b.c0), Fp::add(a.c1, b.c1)}; }
  GM_DEVI static fp2_t sub(const fp2_t &a, const fp2_t &b) { return fp2_t{Fp::sub(a.c0, b.c0), Fp::sub(a.c1, b.c1)}; }
  GM_DEVI static fp2_t dbl(const fp2_t &a) { return add(a, a); }
  GM_DEVI static fp2_t neg(const fp2_t &a) { return fp2_t{Fp::neg(a.c0), Fp::neg(a.c1)}; }
  GM_DEVI static fp2_t mul(const fp2_t &a, const fp2_t &b) {
    const fp_t t0 = Fp::mul(a.c0, b.c0);
    const fp_t t1 = Fp::mul(a.c1, b.c1);
    const fp_t t2 = Fp::mul(Fp::add(a.c0, a.c1), Fp::add(b.c0, b.c1));
    return fp2_t{Fp::sub(t0, t1), Fp::sub(Fp::sub(t2, t0), t1)};
  }
  GM_DEVI static fp2_t sqr(const fp2_t &a) {
    const fp_t s = Fp::add(a.c0, a.c1);
    const fp_t d = Fp::sub(a.c0, a.c1);
    const fp_t m = Fp::mul(a.c0, a.c1);
    return fp2_t{Fp::mul(s, d), Fp::add(m, m)};
  }
  GM_DEVI static fp2_t small(uint32_t k) { return fp2_t{Fp::small(k), Fp::zero()}; }
  // (a0 + a1 i)^-1 = (a0 - a1 i) / (a0^2 + a1^2)  (src/fp2.cu:232)
  __device__ static fp2_t inv(const fp2_t &a) {
    const fp_t n = Fp::add(Fp::sqr(a.c0), Fp::sqr(a.c1));
    const fp_t ni = Fp::inv(n);
    return fp2_t{Fp::mul(a.c0, ni), Fp::mul(Fp::neg(a.c1), ni)};
  }
};

}  // namespace gm
