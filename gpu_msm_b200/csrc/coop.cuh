// Cooperative point operations for the latency-bound phases (upper
// reduction levels, reduction tree, fix-up of long bucket runs, window
// combination): the lane-group size and the operations per group.  Both
// groups use quads (xyzz_quad.cuh).  A 16-lane G2 variant (three Karatsuba Fp
// products of each of the level's four Fp2 products on separate lanes) was
// measured slower on B200: four times the threads at the same register
// footprint pushed the upper levels into a second wave (G2 2^18 reduction
// 5.2 ms against 3.0 ms).
#pragma once
#include "field_f64.cuh"
#include "xyzz_quad.cuh"

namespace gm {

// Cooperative point operations per group (quads for both groups).
template <class F>
struct Coop;
// Build switch: G1 quads on FP64-pipe products (field_f64.cuh).  Off by
// default; on (with GM_OOL_F64), the G1 2^20 reduction measured 1.85 ms
// against 2.03 ms.
#ifndef GM_COOP_F64
#define GM_COOP_F64 0
#endif
template <>
struct Coop<Fp> {
#if GM_COOP_F64
  using A = FpOutF64;
#else
  using A = FpOut;
#endif
  static constexpr int LANES = 4;
  GM_DEVI static void add(xyzz_t<A> &acc, const xyzz_t<A> &o) { q_add<A>(acc, o); }
  GM_DEVI static void dbl(xyzz_t<A> &p) { q_dbl<A>(p); }
};
template <>
struct Coop<Fp2> {
  using A = Fp2Call;
  static constexpr int LANES = 4;
  GM_DEVI static void add(xyzz_t<A> &acc, const xyzz_t<A> &o) { q_add<A>(acc, o); }
  GM_DEVI static void dbl(xyzz_t<A> &p) { q_dbl<A>(p); }
};

// r = k * p for a small non-negative integer k (MSB-first double-and-add)
template <class F>
GM_DEVI void coop_mul_small(xyzz_t<typename Coop<F>::A> &r, const xyzz_t<typename Coop<F>::A> &p, uint32_t k) {
  xyzz_set_inf(r);
  if (k == 0 || xyzz_is_inf(p)) return;
  for (int b = 31 - __clz(k); b >= 0; b--) {
    Coop<F>::dbl(r);
    if ((k >> b) & 1u) Coop<F>::add(r, p);
  }
}

// lane 0 of the calling thread's group
template <class F>
GM_DEVI bool coop_leader() {
  return (threadIdx.x & (Coop<F>::LANES - 1)) == 0;
}

}  // namespace gm
