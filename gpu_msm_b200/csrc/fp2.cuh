// Fp2 = Fp[i]/(i^2 + 1) on sm_100a (pdroalves/gpu_msm include/fp2.h:7,
// non-residue i as in src/fp2.cu:283-294).  Layout {c0, c1} is
// byte-identical to the reference's `Fp2{Fp c0, c1}` (include/fp2.h:10).
//
// Multiplication is 3-mul Karatsuba (the algorithm of src/fp2.cu:88-112):
//   t0 = a0*b0, t1 = a1*b1, t2 = (a0+a1)*(b0+b1); c0 = t0 - t1, c1 = t2 - t0 - t1,
// with the operand sums left unreduced (below 2p, see add_lazy).
// Squaring uses the complex method: c0 = (a0+a1)(a0-a1), c1 = 2*a0*a1.
// Every result is the canonical element, so outputs match the reference's
// fp2_mont_mul bit for bit.
#pragma once
#include "field.cuh"

namespace gm {

struct fp2_t {
  fp_t c0, c1;
};

// Fp2 over a base-field policy B (Fp, or FpOut for an out-of-line product).
// a + b without the final reduction (< 2p for canonical inputs).  Only used
// for Montgomery-product operands: with inputs below 2p the product is below
// 2p before its conditional subtraction (4p < R = 2^448), so its result is
// still canonical.
GM_DEVI fp_t add_lazy(const fp_t &a, const fp_t &b) {
  fp_t r;
  r.v[0] = add_cc(a.v[0], b.v[0]);
#pragma unroll
  for (int i = 1; i < NL; i++) r.v[i] = addc_cc(a.v[i], b.v[i]);
  return r;
}

template <class B>
struct Fp2T {
  using T = fp2_t;
  static constexpr int LIMBS = 2 * NL;

  GM_DEVI static fp2_t zero() { return fp2_t{B::zero(), B::zero()}; }
  GM_DEVI static fp2_t one() { return fp2_t{B::one(), B::zero()}; }
  GM_DEVI static bool is_zero(const fp2_t &a) { return B::is_zero(a.c0) && B::is_zero(a.c1); }
  GM_DEVI static bool is_zero_raw(const fp2_t &a) { return B::is_zero_raw(a.c0) && B::is_zero_raw(a.c1); }
  GM_DEVI static bool eq(const fp2_t &a, const fp2_t &b) { return B::eq(a.c0, b.c0) && B::eq(a.c1, b.c1); }
  GM_DEVI static fp2_t add(const fp2_t &a, const fp2_t &b) { return fp2_t{B::add(a.c0, b.c0), B::add(a.c1, b.c1)}; }
  GM_DEVI static fp2_t sub(const fp2_t &a, const fp2_t &b) { return fp2_t{B::sub(a.c0, b.c0), B::sub(a.c1, b.c1)}; }
  GM_DEVI static fp2_t dbl(const fp2_t &a) { return add(a, a); }
  GM_DEVI static fp2_t neg(const fp2_t &a) { return fp2_t{B::neg(a.c0), B::neg(a.c1)}; }
  GM_DEVI static fp2_t mul(const fp2_t &a, const fp2_t &b) {
    const fp_t t0 = B::mul(a.c0, b.c0);
    const fp_t t1 = B::mul(a.c1, b.c1);
    const fp_t t2 = B::mul(add_lazy(a.c0, a.c1), add_lazy(b.c0, b.c1));
    return fp2_t{B::sub(t0, t1), B::sub(B::sub(t2, t0), t1)};
  }
  GM_DEVI static fp2_t sqr(const fp2_t &a) {
    const fp_t s = add_lazy(a.c0, a.c1);
    const fp_t d = B::sub(a.c0, a.c1);
    const fp_t m = B::mul(a.c0, a.c1);
    return fp2_t{B::mul(s, d), B::add(m, m)};
  }
  GM_DEVI static fp2_t small(uint32_t k) { return fp2_t{B::small(k), B::zero()}; }
  // (a0 + a1 i)^-1 = (a0 - a1 i) / (a0^2 + a1^2)  (src/fp2.cu:232)
  __device__ static fp2_t inv(const fp2_t &a) {
    const fp_t n = B::add(B::sqr(a.c0), B::sqr(a.c1));
    const fp_t ni = B::inv(n);
    return fp2_t{B::mul(a.c0, ni), B::mul(B::neg(a.c1), ni)};
  }
};

using Fp2 = Fp2T<Fp>;
using Fp2Out = Fp2T<FpOut>;

// Fp2 with the whole Fp2 product out of line (one call per Fp2 product):
// the caller keeps no Karatsuba temporaries live across the three Fp
// products, which keeps the G2 accumulation loop within the register file.
static __device__ __noinline__ fp2_t fp2_mul_call(fp2_t a, fp2_t b) { return Fp2Out::mul(a, b); }
static __device__ __noinline__ fp2_t fp2_sqr_call(fp2_t a) { return Fp2Out::sqr(a); }
struct Fp2Call : Fp2Out {
  GM_DEVI static fp2_t mul(const fp2_t &a, const fp2_t &b) { return fp2_mul_call(a, b); }
  GM_DEVI static fp2_t sqr(const fp2_t &a) { return fp2_sqr_call(a); }
};

}  // namespace gm
