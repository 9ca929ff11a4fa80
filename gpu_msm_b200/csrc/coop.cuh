// Cooperative point operations for the latency-bound phases (upper
// reduction levels, reduction tree, fix-up of long bucket runs, window
// combination): the lane-group size and the operations per group.  Both
// groups use quads (xyzz_quad.cuh).  These phases run about one warp per SM
// sub-partition, and such a warp is bound by its own instruction issue, so
// wider groups do not help: a G2 variant on 16 lanes with the three
// Karatsuba Fp products of every Fp2 product on separate lanes issues more
// instructions per addition (16 lanes x 4 products plus the gathers, against
// 4 lanes x 12 products) and measured slower on B200 (G2 2^18 level 1
// 2.46 ms against 1.2 ms on quads).
#pragma once
#include "xyzz_quad.cuh"

namespace gm {

// Cooperative point operations per group (quads for both groups).
template <class F>
struct Coop;
template <>
struct Coop<Fp> {
  using A = FpOut;
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
