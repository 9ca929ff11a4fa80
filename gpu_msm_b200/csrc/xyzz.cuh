// Short-Weierstrass (a = 0) point arithmetic in XYZZ coordinates for the
// bucket method: x = X/ZZ, y = Y/ZZZ with ZZ^3 = ZZZ^2; the point at infinity
// is ZZ = ZZZ = 0.  Formulas from the Explicit-Formulas Database, "xyzz"
// family for a = 0:
//   madd-2008-s  mixed add   (8M + 2S)   bucket += affine base
//   add-2008-s   full add    (12M + 2S)  bucket reduction
//   dbl-2008-s-1 doubling    (6M + 3S)   window combination
//   mdbl-2008-s-1 affine doubling        exception path of madd
// Every addition handles the exceptional inputs the reference's projective
// add handles (src/curve.cu:444-519): infinity operands, P == Q (falls back to
// doubling) and P == -Q (infinity).
#pragma once
#include "fp2.cuh"

namespace gm {

template <class F>
struct xyzz_t {
  typename F::T X, Y, ZZ, ZZZ;
};

template <class F>
struct aff_t {
  typename F::T x, y;
};

template <class F>
GM_DEVI void xyzz_set_inf(xyzz_t<F> &p) {
  p.X = F::zero();
  p.Y = F::zero();
  p.ZZ = F::zero();
  p.ZZZ = F::zero();
}

template <class F>
GM_DEVI bool xyzz_is_inf(const xyzz_t<F> &p) {
  return F::is_zero_raw(p.ZZ);
}

// r = 2*(x, y) for an affine point (mdbl-2008-s-1)
template <class F>
GM_DEVI void xyzz_mdbl(xyzz_t<F> &r, const typename F::T &x, const typename F::T &y) {
  using T = typename F::T;
  if (F::is_zero_raw(y)) {  // 2-torsion: 2P = O
    xyzz_set_inf(r);
    return;
  }
  const T U = F::dbl(y);
  const T V = F::sqr(U);
  const T W = F::mul(U, V);
  const T S = F::mul(x, V);
  const T xx = F::sqr(x);
  const T M = F::add(F::dbl(xx), xx);
  const T X3 = F::sub(F::sqr(M), F::dbl(S));
  const T Y3 = F::sub(F::mul(M, F::sub(S, X3)), F::mul(W, y));
  r.X = X3;
  r.Y = Y3;
  r.ZZ = V;
  r.ZZZ = W;
}

// r = 2*p (dbl-2008-s-1)
template <class F>
GM_DEVI void xyzz_dbl(xyzz_t<F> &r, const xyzz_t<F> &p) {
  using T = typename F::T;
  if (xyzz_is_inf(p)) {
    r = p;
    return;
  }
  const T U = F::dbl(p.Y);
  const T V = F::sqr(U);
  const T W = F::mul(U, V);
  const T S = F::mul(p.X, V);
  const T xx = F::sqr(p.X);
  const T M = F::add(F::dbl(xx), xx);
  const T X3 = F::sub(F::sqr(M), F::dbl(S));
  const T Y3 = F::sub(F::mul(M, F::sub(S, X3)), F::mul(W, p.Y));
  const T ZZ3 = F::mul(V, p.ZZ);
  const T ZZZ3 = F::mul(W, p.ZZZ);
  r.X = X3;
  r.Y = Y3;
  r.ZZ = ZZ3;
  r.ZZZ = ZZZ3;
}

template <class F>
__device__ __noinline__ void xyzz_mdbl_cold(xyzz_t<F> &r, const typename F::T &x, const typename F::T &y) {
  xyzz_mdbl<F>(r, x, y);
}
template <class F>
__device__ __noinline__ void xyzz_dbl_exc(xyzz_t<F> &p) {
  xyzz_dbl<F>(p, p);
}

// acc += (x2, y2) (madd-2008-s).  The products are ordered so that few
// values are live at once (each value dies at its last use), which keeps
// the Fp2 form within the register file.  The affine point comes from a
// provider with x() and y(): registers (RegPoint), or a shared-memory stage
// read at first use, so that the point is not held in registers across the
// out-of-line products.
template <class F>
struct RegPoint {
  const typename F::T &x_, &y_;
  GM_DEVI const typename F::T &x() const { return x_; }
  GM_DEVI const typename F::T &y() const { return y_; }
};

template <class F, class PT>
GM_DEVI void xyzz_madd_pt(xyzz_t<F> &acc, const PT &pt) {
  using T = typename F::T;
  if (xyzz_is_inf(acc)) {
    acc.X = pt.x();
    acc.Y = pt.y();
    acc.ZZ = F::one();
    acc.ZZZ = F::one();
    return;
  }
  const T P = F::sub(F::mul(pt.x(), acc.ZZ), acc.X);    // U2 - X1
  const T R = F::sub(F::mul(pt.y(), acc.ZZZ), acc.Y);   // S2 - Y1
  if (F::is_zero(P)) {
    if (F::is_zero(R))
      xyzz_mdbl_cold<F>(acc, pt.x(), pt.y());
    else
      xyzz_set_inf(acc);
    return;
  }
  const T PP = F::sqr(P);
  acc.ZZ = F::mul(acc.ZZ, PP);
  const T PPP = F::mul(P, PP);
  acc.ZZZ = F::mul(acc.ZZZ, PPP);
  const T Q = F::mul(acc.X, PP);
  const T X3 = F::sub(F::sub(F::sqr(R), PPP), F::dbl(Q));
  acc.Y = F::sub(F::mul(R, F::sub(Q, X3)), F::mul(acc.Y, PPP));
  acc.X = X3;
}

template <class F>
GM_DEVI void xyzz_madd(xyzz_t<F> &acc, const typename F::T &x2, const typename F::T &y2) {
  xyzz_madd_pt<F>(acc, RegPoint<F>{x2, y2});
}

// acc += q (add-2008-s)
template <class F>
GM_DEVI void xyzz_add(xyzz_t<F> &acc, const xyzz_t<F> &q) {
  using T = typename F::T;
  if (xyzz_is_inf(q)) return;
  if (xyzz_is_inf(acc)) {
    acc = q;
    return;
  }
  const T U1 = F::mul(acc.X, q.ZZ);
  const T U2 = F::mul(q.X, acc.ZZ);
  const T S1 = F::mul(acc.Y, q.ZZZ);
  const T S2 = F::mul(q.Y, acc.ZZZ);
  const T P = F::sub(U2, U1);
  const T R = F::sub(S2, S1);
  if (F::is_zero(P)) {
    if (F::is_zero(R))
      xyzz_dbl_exc<F>(acc);
    else
      xyzz_set_inf(acc);
    return;
  }
  const T PP = F::sqr(P);
  const T PPP = F::mul(P, PP);
  const T Q = F::mul(U1, PP);
  const T X3 = F::sub(F::sub(F::sqr(R), PPP), F::dbl(Q));
  const T Y3 = F::sub(F::mul(R, F::sub(Q, X3)), F::mul(S1, PPP));
  acc.ZZ = F::mul(F::mul(acc.ZZ, q.ZZ), PP);
  acc.ZZZ = F::mul(F::mul(acc.ZZZ, q.ZZZ), PPP);
  acc.X = X3;
  acc.Y = Y3;
}

// XYZZ -> homogeneous projective (X*ZZZ, Y*ZZ, ZZ*ZZZ): x = X'/Z', y = Y'/Z'.
// Infinity maps to (0, 0, 0) like g1_projective_point_at_infinity
// (src/curve.cu:740).
template <class F>
GM_DEVI void xyzz_to_proj(typename F::T &X, typename F::T &Y, typename F::T &Z, const xyzz_t<F> &p) {
  if (xyzz_is_inf(p)) {
    X = F::zero();
    Y = F::zero();
    Z = F::zero();
    return;
  }
  X = F::mul(p.X, p.ZZZ);
  Y = F::mul(p.Y, p.ZZ);
  Z = F::mul(p.ZZ, p.ZZZ);
}

// homogeneous projective -> XYZZ: x = X/Z, y = Y/Z -> (X*Z, Y*Z^2, Z^2, Z^3)
template <class F>
GM_DEVI void proj_to_xyzz(xyzz_t<F> &r, const typename F::T &X, const typename F::T &Y, const typename F::T &Z) {
  if (F::is_zero(Z)) {
    xyzz_set_inf(r);
    return;
  }
  const typename F::T Z2 = F::sqr(Z);
  r.ZZ = Z2;
  r.ZZZ = F::mul(Z2, Z);
  r.X = F::mul(X, Z);
  r.Y = F::mul(Y, Z2);
}

// Out-of-line copies for kernels off the accumulation hot loop (fix-up,
// bucket reduction, window combination, exception paths): one call site each
// keeps code size and compile time bounded.  The accumulation loop inlines
// xyzz_madd directly.
template <class F>
__device__ __noinline__ void xyzz_add_cold(xyzz_t<F> &acc, const xyzz_t<F> &q) {
  xyzz_add<F>(acc, q);
}
template <class F>
__device__ __noinline__ void xyzz_dbl_cold(xyzz_t<F> &p) {
  xyzz_dbl<F>(p, p);
}

}  // namespace gm
