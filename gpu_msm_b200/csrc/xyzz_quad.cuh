// XYZZ point arithmetic spread over a quad: four consecutive lanes of a warp
// that hold the same operands and produce the same results.  Each field
// product of a formula is computed by one lane of the quad and broadcast to
// the other three with shuffles, so an addition (add-2008-s, 12M + 2S) has a
// serial depth of 4 products and a doubling (dbl-2008-s-1, 6M + 3S) of 3,
// against 14 and 9 in one thread.
//
// Why: one Montgomery product is a single carry chain of ~800 dependent
// IMADs (about 2,900 cycles for one thread on B200), and two independent
// products in one thread do not overlap, because the PTX carry flag orders
// them.  Where there are too few independent additions to fill the GPU --
// the upper levels of the bucket reduction, the fix-up of long bucket runs,
// the window combination -- only more lanes per addition shorten the time.
//
// Contract: all four lanes of a quad call these functions together with
// equal arguments; every branch inside depends only on quad-uniform values.
// Blocks are one-dimensional with a multiple of 32 threads, so the quad of a
// thread is lanes (threadIdx.x & ~3) .. +3 of its warp.
#pragma once
#include "xyzz.cuh"

namespace gm {

GM_DEVI unsigned quad_mask() { return 0xFu << (threadIdx.x & 28u); }
GM_DEVI int quad_lane() { return (int)(threadIdx.x & 3u); }

GM_DEVI fp_t q_bcast(const fp_t &v, int src, unsigned mask) {
  fp_t r;
#pragma unroll
  for (int i = 0; i < NL; i++) r.v[i] = __shfl_sync(mask, v.v[i], src, 4);
  return r;
}
GM_DEVI fp2_t q_bcast(const fp2_t &v, int src, unsigned mask) {
  return fp2_t{q_bcast(v.c0, src, mask), q_bcast(v.c1, src, mask)};
}

// operand of lane q among four candidates
GM_DEVI fp_t q_pick(int q, const fp_t &a0, const fp_t &a1, const fp_t &a2, const fp_t &a3) {
  fp_t r;
#pragma unroll
  for (int i = 0; i < NL; i++) r.v[i] = q == 0 ? a0.v[i] : q == 1 ? a1.v[i] : q == 2 ? a2.v[i] : a3.v[i];
  return r;
}
GM_DEVI fp2_t q_pick(int q, const fp2_t &a0, const fp2_t &a1, const fp2_t &a2, const fp2_t &a3) {
  return fp2_t{q_pick(q, a0.c0, a1.c0, a2.c0, a3.c0), q_pick(q, a0.c1, a1.c1, a2.c1, a3.c1)};
}

// p = 2p (dbl-2008-s-1).  Depth: {V = U^2, xx = X^2} -> {W = U V, S = X V,
// M^2, ZZ V} -> {M (S - X3), W Y, ZZZ W}.
template <class F>
__device__ __noinline__ void q_dbl(xyzz_t<F> &p) {
  using T = typename F::T;
  if (xyzz_is_inf(p)) return;
  const int q = quad_lane();
  const unsigned m = quad_mask();
  const T U = F::dbl(p.Y);
  T r = F::mul(q_pick(q, U, p.X, U, p.X), q_pick(q, U, p.X, U, p.X));
  const T V = q_bcast(r, 0, m), xx = q_bcast(r, 1, m);
  const T M = F::add(F::dbl(xx), xx);
  r = F::mul(q_pick(q, U, p.X, M, V), q_pick(q, V, V, M, p.ZZ));
  const T W = q_bcast(r, 0, m), S = q_bcast(r, 1, m), MM = q_bcast(r, 2, m), ZZ3 = q_bcast(r, 3, m);
  const T X3 = F::sub(MM, F::dbl(S));
  r = F::mul(q_pick(q, M, W, W, M), q_pick(q, F::sub(S, X3), p.Y, p.ZZZ, S));
  const T Y3a = q_bcast(r, 0, m), WY = q_bcast(r, 1, m), ZZZ3 = q_bcast(r, 2, m);
  p.X = X3;
  p.Y = F::sub(Y3a, WY);
  p.ZZ = ZZ3;
  p.ZZZ = ZZZ3;
}

// acc += o (add-2008-s), same exceptional cases as xyzz_add: an infinite
// operand, P == Q (doubling) and P == -Q (infinity).  Depth: {U1, U2, S1, S2}
// -> {P^2, R^2, ZZ1 ZZ2, ZZZ1 ZZZ2} -> {P PP, U1 PP, ZZ12 PP}
// -> {R (Q - X3), S1 PPP, ZZZ12 PPP}.
template <class F>
__device__ __noinline__ void q_add(xyzz_t<F> &acc, const xyzz_t<F> &o) {
  using T = typename F::T;
  if (xyzz_is_inf(o)) return;
  if (xyzz_is_inf(acc)) {
    acc = o;
    return;
  }
  const int q = quad_lane();
  const unsigned m = quad_mask();
  T r = F::mul(q_pick(q, acc.X, o.X, acc.Y, o.Y), q_pick(q, o.ZZ, acc.ZZ, o.ZZZ, acc.ZZZ));
  const T U1 = q_bcast(r, 0, m), U2 = q_bcast(r, 1, m), S1 = q_bcast(r, 2, m), S2 = q_bcast(r, 3, m);
  const T P = F::sub(U2, U1);
  const T R = F::sub(S2, S1);
  if (F::is_zero(P)) {
    if (F::is_zero(R))
      q_dbl<F>(acc);
    else
      xyzz_set_inf(acc);
    return;
  }
  r = F::mul(q_pick(q, P, R, acc.ZZ, acc.ZZZ), q_pick(q, P, R, o.ZZ, o.ZZZ));
  const T PP = q_bcast(r, 0, m), RR = q_bcast(r, 1, m), ZZ12 = q_bcast(r, 2, m), ZZZ12 = q_bcast(r, 3, m);
  r = F::mul(q_pick(q, P, U1, ZZ12, P), PP);
  const T PPP = q_bcast(r, 0, m), Qv = q_bcast(r, 1, m), ZZ3 = q_bcast(r, 2, m);
  const T X3 = F::sub(F::sub(RR, PPP), F::dbl(Qv));
  r = F::mul(q_pick(q, R, S1, ZZZ12, R), q_pick(q, F::sub(Qv, X3), PPP, PPP, PPP));
  const T Y3a = q_bcast(r, 0, m), Y3b = q_bcast(r, 1, m), ZZZ3 = q_bcast(r, 2, m);
  acc.X = X3;
  acc.Y = F::sub(Y3a, Y3b);
  acc.ZZ = ZZ3;
  acc.ZZZ = ZZZ3;
}

// r = k * p for a small non-negative integer k (MSB-first double-and-add)
template <class F>
GM_DEVI void q_mul_small(xyzz_t<F> &r, const xyzz_t<F> &p, uint32_t k) {
  xyzz_set_inf(r);
  if (k == 0 || xyzz_is_inf(p)) return;
  for (int b = 31 - __clz(k); b >= 0; b--) {
    q_dbl<F>(r);
    if ((k >> b) & 1u) q_add<F>(r, p);
  }
}

}  // namespace gm
