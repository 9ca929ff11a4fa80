// Single-element field and point operations on device pointers: the C-ABI
// behind the reference's stream APIs fp_*_async (pdroalves/gpu_msm
// include/fp.h:158-204, src/fp_kernels.cu:753-900), fp2_*_async
// (include/fp2.h:99-133, src/fp2_kernels.cu:564-680) and
// point_*_async<G1Point|G2Point> (include/curve.h:156-211,
// src/curve.cu:2288-2500).  cxx_api.cu builds the reference-named C++
// functions and the host-pointer helpers of include/fp_kernels.h and
// include/fp2_kernels.h on these entry points.
//
// Each call is one short kernel on the caller's stream.  The operations are
// exact modular arithmetic, so every correct evaluation gives the canonical
// result the reference computes; the reference's conventions for special
// cases are kept:
//   - fp/fp2 mul, square, inv, div, pow, sqrt take and return standard form
//     (the reference converts to Montgomery form and back inside,
//     src/fp.cu:424, :448-500); here a standard-form product is one
//     Montgomery product followed by a product with R^2, which gives the
//     same value with two products instead of four;
//   - inv(0) = 0 and a / 0 = 0 (src/fp.cu:522, :571; src/fp2.cu:232);
//   - sqrt(a) = a^((p+1)/4) for a quadratic residue (p = 3 mod 4), with the
//     reference's check that the square gives a back (src/fp.cu fp_sqrt);
//   - point add, double and neg are the affine formulas with one
//     Montgomery-form inversion and the reference's branch order
//     (src/curve.cu:72-227), so inputs that share x but are not P and -P
//     give its result too;
//   - scalar multiplication runs MSB-first double-and-add in XYZZ
//     coordinates on one quad (xyzz_quad.cuh) and inverts once at the end:
//     one inversion instead of one per doubling and addition.  For points
//     on the curve the group law makes its result equal to the reference's
//     affine double-and-add (src/curve.cu:230-268).
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/gpu_msm_b200.h"
#include "msm_engine.h"
#include "msm_kernels.cuh"
#include "xyzz_quad.cuh"

namespace {

using gm::fp2_t;
using gm::fp_t;
using gm::NL;

GM_DEVI fp_t r2_const() {
  fp_t r;
#pragma unroll
  for (int i = 0; i < NL; i++) r.v[i] = gm::FpConst::R2(i);
  return r;
}
GM_DEVI fp_t p_const() {
  fp_t r;
#pragma unroll
  for (int i = 0; i < NL; i++) r.v[i] = gm::FpConst::P(i);
  return r;
}
GM_DEVI fp_t one_std() {
  fp_t r = gm::Fp::zero();
  r.v[0] = 1;
  return r;
}

// Montgomery-form Fp with every product out of line: one copy of the
// ~900-instruction product per kernel instead of one per call site keeps
// these single-thread kernels small and quick to compile.
__device__ __noinline__ fp_t f1_inv(fp_t a) {
  // a^(p-2), left-to-right square-and-multiply; 0 -> 0 (src/fp.cu:545)
  fp_t acc;
#pragma unroll
  for (int i = 0; i < NL; i++) acc.v[i] = gm::FpConst::ONE(i);
  for (int w = NL - 1; w >= 0; w--) {
    const uint32_t e = (w == 0) ? gm::FpConst::P(0) - 2u : gm::FpConst::P(w);
    for (int b = 31; b >= 0; b--) {
      acc = gm::fp_sqr_call(acc);
      if ((e >> b) & 1u) acc = gm::fp_mul_call(acc, a);
    }
  }
  return acc;
}
struct F1 : gm::FpOut {
  GM_DEVI static fp_t to_mont(const fp_t &a) { return mul(a, r2_const()); }
  GM_DEVI static fp_t from_mont(const fp_t &a) {
    fp_t o = zero();
    o.v[0] = 1;
    return mul(a, o);
  }
  GM_DEVI static fp_t inv(const fp_t &a) { return f1_inv(a); }
};
using F2 = gm::Fp2T<F1>;  // Montgomery-form Fp2 over F1

// reference-layout (u64 limbs) element <-> registers, and form conversions
GM_DEVI void ld(fp_t &r, const uint64_t *s) { gm::load_ref<gm::Fp>(r, s); }
GM_DEVI void ld(fp2_t &r, const uint64_t *s) { gm::load_ref<gm::Fp2>(r, s); }
GM_DEVI void st(uint64_t *d, fp_t a) { gm::store_ref<gm::Fp>(d, a); }
GM_DEVI void st(uint64_t *d, fp2_t a) { gm::store_ref<gm::Fp2>(d, a); }
GM_DEVI fp_t to_m(const fp_t &a) { return F1::to_mont(a); }
GM_DEVI fp2_t to_m(const fp2_t &a) { return fp2_t{F1::to_mont(a.c0), F1::to_mont(a.c1)}; }
GM_DEVI fp_t from_m(const fp_t &a) { return F1::from_mont(a); }
GM_DEVI fp2_t from_m(const fp2_t &a) { return fp2_t{F1::from_mont(a.c0), F1::from_mont(a.c1)}; }

// limb-wise comparison from the top limb (src/fp.cu fp_cmp)
GM_DEVI int cmp_raw(const fp_t &a, const fp_t &b) {
  for (int i = NL - 1; i >= 0; i--) {
    if (a.v[i] > b.v[i]) return 1;
    if (a.v[i] < b.v[i]) return -1;
  }
  return 0;
}

// ---- standard-form Fp -------------------------------------------------------
// (a b R^-1) R^2 R^-1 = a b
__device__ fp_t std_mul(const fp_t &a, const fp_t &b) { return F1::mul(F1::mul(a, b), r2_const()); }

// a^e for standard-form a; e is nw little-endian 32-bit words, read MSB first
// (the square-and-multiply of src/fp.cu:448-500; e = 0 gives 1)
__device__ fp_t std_pow(const fp_t &a, const uint32_t *e, int nw) {
  const fp_t am = F1::to_mont(a);
  fp_t acc = F1::one();
  for (int w = nw - 1; w >= 0; w--)
    for (int b = 31; b >= 0; b--) {
      acc = F1::sqr(acc);
      if ((e[w] >> b) & 1u) acc = F1::mul(acc, am);
    }
  return F1::from_mont(acc);
}

// e = (p >> s) + add: (p-1)/2 = p >> 1 (p odd) and (p+1)/4 = (p >> 2) + 1
// (p = 3 mod 4)
GM_DEVI void p_exponent(uint32_t *e, int s, uint32_t add) {
#pragma unroll
  for (int i = 0; i < NL; i++) {
    const uint32_t hi = i + 1 < NL ? gm::FpConst::P(i + 1) : 0u;
    e[i] = (gm::FpConst::P(i) >> s) | (hi << (32 - s));
  }
  uint32_t c = add;
  for (int i = 0; i < NL; i++) {
    const uint32_t t = e[i] + c;
    c = t < c ? 1u : 0u;
    e[i] = t;
  }
}

__device__ fp_t std_inv(const fp_t &a) {
  if (F1::is_zero_raw(a)) return F1::zero();
  return F1::from_mont(F1::inv(F1::to_mont(a)));
}

// Euler's criterion, 0 counts as a residue (src/fp.cu fp_is_quadratic_residue)
__device__ bool std_is_qr(const fp_t &a) {
  if (F1::is_zero_raw(a)) return true;
  uint32_t e[NL];
  p_exponent(e, 1, 0u);
  return F1::eq(std_pow(a, e, NL), one_std());
}

// src/fp.cu fp_sqrt: a^((p+1)/4), then the reference's two checks
__device__ bool std_sqrt(fp_t &c, const fp_t &a) {
  if (F1::is_zero_raw(a)) {
    c = F1::zero();
    return true;
  }
  if (!std_is_qr(a)) {
    c = F1::zero();
    return false;
  }
  uint32_t e[NL];
  p_exponent(e, 2, 1u);
  c = std_pow(a, e, NL);
  if (F1::eq(std_mul(c, c), a)) return true;
  const fp_t alt = F1::sub(p_const(), c);
  if (F1::eq(std_mul(alt, alt), a)) {
    c = alt;
    return true;
  }
  return false;
}

// ---- standard-form Fp2 ------------------------------------------------------
GM_DEVI fp2_t to_r(const fp2_t &a) { return fp2_t{F1::mul(a.c0, r2_const()), F1::mul(a.c1, r2_const())}; }
__device__ fp2_t std2_mul(const fp2_t &a, const fp2_t &b) { return to_r(F2::mul(a, b)); }
__device__ fp2_t std2_sqr(const fp2_t &a) { return to_r(F2::sqr(a)); }
__device__ fp2_t std2_inv(const fp2_t &a) {
  if (F2::is_zero_raw(a)) return F2::zero();
  const fp2_t m{F1::to_mont(a.c0), F1::to_mont(a.c1)};
  const fp2_t i = F2::inv(m);
  return fp2_t{F1::from_mont(i.c0), F1::from_mont(i.c1)};
}

// ---- element kernels (one thread) ------------------------------------------
__global__ void k_fp_elem(int op, uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t arg,
                          int32_t *flag) {
  fp_t x = F1::zero(), y = F1::zero(), z = F1::zero();
  if (a) ld(x, a);
  if (b) ld(y, b);
  int32_t f = 0;
  bool write = true;
  switch (op) {
    case GM_FP_ADD: z = F1::add(x, y); break;
    case GM_FP_SUB: z = F1::sub(x, y); break;
    case GM_FP_MUL: z = std_mul(x, y); break;
    case GM_FP_NEG: z = F1::neg(x); break;
    case GM_FP_INV: z = std_inv(x); break;
    case GM_FP_DIV: z = F1::is_zero_raw(y) ? F1::zero() : std_mul(x, std_inv(y)); break;
    case GM_FP_COPY: z = x; break;
    case GM_FP_ZERO: z = F1::zero(); break;
    case GM_FP_ONE: z = one_std(); break;
    case GM_FP_TO_MONT: z = F1::to_mont(x); break;
    case GM_FP_FROM_MONT: z = F1::from_mont(x); break;
    case GM_FP_MONT_MUL: z = F1::mul(x, y); break;
    case GM_FP_CMP: f = cmp_raw(x, y); write = false; break;
    case GM_FP_IS_ZERO: f = F1::is_zero_raw(x); write = false; break;
    case GM_FP_IS_ONE: f = F1::eq(x, one_std()); write = false; break;
    case GM_FP_CMOV:
      write = (arg & 1u) != 0;
      z = x;
      break;
    case GM_FP_SQRT: f = std_sqrt(z, x); break;
    case GM_FP_IS_QR: f = std_is_qr(x); write = false; break;
    case GM_FP_POW_U64: {
      const uint32_t e[2] = {(uint32_t)arg, (uint32_t)(arg >> 32)};
      z = std_pow(x, e, 2);
      break;
    }
    default: write = false; break;
  }
  if (write) st(c, z);
  if (flag) *flag = f;
}

__global__ void k_fp2_elem(int op, uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t arg,
                           int32_t *flag) {
  fp2_t x = F2::zero(), y = F2::zero(), z = F2::zero();
  if (a) ld(x, a);
  if (b) ld(y, b);
  int32_t f = 0;
  bool write = true;
  switch (op) {
    case GM_FP2_ADD: z = F2::add(x, y); break;
    case GM_FP2_SUB: z = F2::sub(x, y); break;
    case GM_FP2_MUL: z = std2_mul(x, y); break;
    case GM_FP2_SQUARE: z = std2_sqr(x); break;
    case GM_FP2_NEG: z = F2::neg(x); break;
    case GM_FP2_CONJUGATE:
    case GM_FP2_FROBENIUS: z = fp2_t{x.c0, F1::neg(x.c1)}; break;  // src/fp2.cu: a^p = conj(a)
    case GM_FP2_INV: z = std2_inv(x); break;
    case GM_FP2_DIV: z = std2_mul(x, std2_inv(y)); break;
    case GM_FP2_COPY: z = x; break;
    case GM_FP2_MUL_BY_I: z = fp2_t{F1::neg(x.c1), x.c0}; break;
    case GM_FP2_CMP: {
      const int c0 = cmp_raw(x.c0, y.c0);
      f = c0 != 0 ? c0 : cmp_raw(x.c1, y.c1);
      write = false;
      break;
    }
    case GM_FP2_IS_ZERO: f = F2::is_zero_raw(x); write = false; break;
    case GM_FP2_IS_ONE: f = F1::eq(x.c0, one_std()) && F1::is_zero_raw(x.c1); write = false; break;
    case GM_FP2_CMOV:
      write = (arg & 1u) != 0;
      z = x;
      break;
    case GM_FP2_MONT_MUL: z = F2::mul(x, y); break;
    default: write = false; break;
  }
  if (write) st(c, z);
  if (flag) *flag = f;
}

// ---- affine points (Montgomery form), reference layout ----------------------
template <class F>
struct RefPt {
  using T = typename F::T;
  static constexpr int Hw = F::LIMBS / 2;  // u64 words per coordinate
  T x, y;
  bool inf;
  GM_DEVI void load(const uint64_t *p) {
    ld(x, p);
    ld(y, p + Hw);
    inf = reinterpret_cast<const uint8_t *>(p + 2 * Hw)[0] != 0;
  }
  // coordinates and the flag byte; the pad bytes are left as they are
  GM_DEVI void store(uint64_t *p) {
    st(p, x);
    st(p + Hw, y);
    reinterpret_cast<uint8_t *>(p + 2 * Hw)[0] = inf ? 1 : 0;
  }
  GM_DEVI static RefPt infinity() { return RefPt{F::zero(), F::zero(), true}; }
};

// 2P (src/curve.cu:86-117): lambda = 3x^2 / 2y
template <class F>
__device__ RefPt<F> aff_double(const RefPt<F> &p) {
  using T = typename F::T;
  if (p.inf || F::is_zero_raw(p.y)) return RefPt<F>::infinity();
  const T xx = F::mul(p.x, p.x);
  const T t = F::add(F::add(xx, xx), xx);
  const T lam = F::mul(F::inv(F::add(p.y, p.y)), t);
  const T x3 = F::sub(F::mul(lam, lam), F::add(p.x, p.x));
  const T y3 = F::sub(F::mul(lam, F::sub(p.x, x3)), p.y);
  return RefPt<F>{x3, y3, false};
}

// P + Q (src/curve.cu:173-227), same branch order
template <class F>
__device__ RefPt<F> aff_add(const RefPt<F> &p, const RefPt<F> &q) {
  using T = typename F::T;
  if (p.inf) return q;
  if (q.inf) return p;
  const bool same_x = F::eq(p.x, q.x);
  if (same_x && F::eq(p.y, F::neg(q.y))) return RefPt<F>::infinity();
  if (same_x && F::eq(p.y, q.y)) return aff_double<F>(p);
  const T lam = F::mul(F::inv(F::sub(q.x, p.x)), F::sub(q.y, p.y));
  const T x3 = F::sub(F::sub(F::mul(lam, lam), p.x), q.x);
  const T y3 = F::sub(F::mul(lam, F::sub(p.x, x3)), p.y);
  return RefPt<F>{x3, y3, false};
}

// one thread: everything but the scalar multiplications
template <class F>
__global__ void k_point_elem(int op, uint64_t *r, const uint64_t *p, const uint64_t *q) {
  RefPt<F> a, b, out;
  if (p) a.load(p);
  if (q) b.load(q);
  switch (op) {
    case GM_PT_ADD: out = aff_add<F>(a, b); break;
    case GM_PT_DOUBLE: out = aff_double<F>(a); break;
    case GM_PT_NEG:  // src/curve.cu:72-82
      out = a.inf ? RefPt<F>::infinity() : RefPt<F>{a.x, F::neg(a.y), false};
      break;
    case GM_PT_TO_MONT:  // src/curve.cu:2313-2325
      out = a.inf ? RefPt<F>::infinity()
                  : RefPt<F>{to_m(a.x), to_m(a.y), false};
      break;
    case GM_PT_FROM_MONT:  // src/curve.cu:2328-2340
      out = a.inf ? RefPt<F>::infinity()
                  : RefPt<F>{from_m(a.x), from_m(a.y), false};
      break;
    case GM_PT_AT_INFINITY: out = RefPt<F>::infinity(); break;
    default: return;
  }
  out.store(r);
}

// k * P, one warp: each quad runs the same double-and-add over the scalar
// bits (MSB first) with the quad-parallel XYZZ formulas; lane 0 stores.
// `scalar` holds `limbs` u64 limbs; when it is null the scalar is k64.
template <class F>
__global__ void k_point_smul(uint64_t *r, const uint64_t *p, const uint64_t *scalar, int limbs, uint64_t k64) {
  using T = typename F::T;
  RefPt<F> a;
  a.load(p);
  gm::xyzz_t<F> acc;
  gm::xyzz_set_inf(acc);
  if (!a.inf) {
    gm::xyzz_t<F> base;
    base.X = a.x;
    base.Y = a.y;
    base.ZZ = F::one();
    base.ZZZ = F::one();
    const int nl = scalar ? limbs : 1;
    for (int l = nl - 1; l >= 0; l--) {
      const uint64_t w = scalar ? scalar[l] : k64;
      for (int bit = 63; bit >= 0; bit--) {
        gm::q_dbl<F>(acc);
        if ((w >> bit) & 1u) gm::q_add<F>(acc, base);
      }
    }
  }
  RefPt<F> out = RefPt<F>::infinity();
  if (!gm::xyzz_is_inf(acc)) {
    // x = X / ZZ = X ZZZ I, y = Y / ZZZ = Y ZZ I with I = 1 / (ZZ ZZZ)
    const T I = F::inv(F::mul(acc.ZZ, acc.ZZZ));
    out = RefPt<F>{F::mul(acc.X, F::mul(I, acc.ZZZ)), F::mul(acc.Y, F::mul(I, acc.ZZ)), false};
  }
  if (threadIdx.x == 0) out.store(r);
}

// ok[i] = 1 when point i (affine, Montgomery form) satisfies
// y^2 = x^3 + b or carries the infinity flag, else 0.  b is the constant the
// reference's generators satisfy: 1 for G1, 1 + i for G2.  (The reference's
// is_on_curve_g1/g2, src/curve.cu:280-360, use b = 4 and b' = 4i, which its
// own generators do not satisfy; nothing on its MSM path reads them.)
template <class F>
__global__ void k_on_curve(const uint64_t *__restrict__ pts, int64_t n, uint8_t *__restrict__ ok) {
  constexpr int WORDS = 2 * RefPt<F>::Hw + 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    RefPt<F> p;
    p.load(pts + i * WORDS);
    bool good = p.inf;
    if (!good) {
      typename F::T b = F::one();  // 1 (G1); 1 + i (G2) below
      if constexpr (F::LIMBS == 2 * NL) b.c1 = F1::one();
      const typename F::T rhs = F::add(F::mul(F::mul(p.x, p.x), p.x), b);
      good = F::eq(F::mul(p.y, p.y), rhs);
    }
    ok[i] = good ? 1 : 0;
  }
}

int launched(const char *what) {
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, what);
}

int bad_arg(const char *msg) {
  gm::set_last_error(msg);
  return gm::GM_ERR_ARG;
}

// operand needs of the field ops: bit 0 = c, 1 = a, 2 = b, 3 = flag
int fp_needs(int op) {
  switch (op) {
    case GM_FP_ADD:
    case GM_FP_SUB:
    case GM_FP_MUL:
    case GM_FP_DIV:
    case GM_FP_MONT_MUL: return 7;
    case GM_FP_NEG:
    case GM_FP_INV:
    case GM_FP_COPY:
    case GM_FP_TO_MONT:
    case GM_FP_FROM_MONT:
    case GM_FP_CMOV:
    case GM_FP_POW_U64: return 3;
    case GM_FP_ZERO:
    case GM_FP_ONE: return 1;
    case GM_FP_CMP: return 14;
    case GM_FP_IS_ZERO:
    case GM_FP_IS_ONE:
    case GM_FP_IS_QR: return 10;
    case GM_FP_SQRT: return 11;
    default: return -1;
  }
}

int fp2_needs(int op) {
  switch (op) {
    case GM_FP2_ADD:
    case GM_FP2_SUB:
    case GM_FP2_MUL:
    case GM_FP2_DIV:
    case GM_FP2_MONT_MUL: return 7;
    case GM_FP2_SQUARE:
    case GM_FP2_NEG:
    case GM_FP2_CONJUGATE:
    case GM_FP2_INV:
    case GM_FP2_COPY:
    case GM_FP2_MUL_BY_I:
    case GM_FP2_FROBENIUS:
    case GM_FP2_CMOV: return 3;
    case GM_FP2_CMP: return 14;
    case GM_FP2_IS_ZERO:
    case GM_FP2_IS_ONE: return 10;
    default: return -1;
  }
}

int check_needs(int needs, const void *c, const void *a, const void *b, const void *flag) {
  if (needs < 0) return bad_arg("unknown element op");
  if (((needs & 1) && !c) || ((needs & 2) && !a) || ((needs & 4) && !b) || ((needs & 8) && !flag))
    return bad_arg("element op: null pointer argument");
  return gm::GM_OK;
}

template <class F>
int point_elem(gm_stream_t stream, uint32_t gpu_index, int op, void *d_r, const void *d_p, const void *d_q,
               const uint64_t *d_scalar, int scalar_limbs, uint64_t scalar_u64) {
  if (op < 0 || op >= GM_PT_OP_COUNT) return bad_arg("unknown point op");
  if (!d_r) return bad_arg("point op: null result pointer");
  if (op != GM_PT_AT_INFINITY && !d_p) return bad_arg("point op: null point argument");
  if (op == GM_PT_ADD && !d_q) return bad_arg("point op: null point argument");
  if (op == GM_PT_SCALAR_MUL && scalar_limbs > 0 && !d_scalar) return bad_arg("point op: null scalar");
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (op == GM_PT_SCALAR_MUL || op == GM_PT_SCALAR_MUL_U64) {
    // a scalar of no limbs is zero (src/curve.cu:240-249): pass one zero word
    const bool limbs_given = op == GM_PT_SCALAR_MUL && scalar_limbs > 0;
    k_point_smul<F><<<1, 32, 0, s>>>((uint64_t *)d_r, (const uint64_t *)d_p, limbs_given ? d_scalar : nullptr,
                                     limbs_given ? scalar_limbs : 1,
                                     op == GM_PT_SCALAR_MUL_U64 ? scalar_u64 : 0ull);
    return launched("k_point_smul");
  }
  k_point_elem<F><<<1, 1, 0, s>>>(op, (uint64_t *)d_r, (const uint64_t *)d_p, (const uint64_t *)d_q);
  return launched("k_point_elem");
}

}  // namespace

extern "C" {

int gm_fp_elem(gm_stream_t stream, uint32_t gpu_index, int op, Fp *d_c, const Fp *d_a, const Fp *d_b, uint64_t arg,
               int32_t *d_flag) {
  int rc = check_needs(fp_needs(op), d_c, d_a, d_b, d_flag);
  if (rc) return rc;
  rc = gm::select_device(gpu_index);
  if (rc) return rc;
  const int needs = fp_needs(op);
  k_fp_elem<<<1, 1, 0, (cudaStream_t)stream>>>(op, (needs & 1) ? (uint64_t *)d_c : nullptr,
                                               (needs & 2) ? (const uint64_t *)d_a : nullptr,
                                               (needs & 4) ? (const uint64_t *)d_b : nullptr, arg,
                                               (needs & 8) ? d_flag : nullptr);
  return launched("k_fp_elem");
}

int gm_fp2_elem(gm_stream_t stream, uint32_t gpu_index, int op, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b,
                uint64_t arg, int32_t *d_flag) {
  int rc = check_needs(fp2_needs(op), d_c, d_a, d_b, d_flag);
  if (rc) return rc;
  rc = gm::select_device(gpu_index);
  if (rc) return rc;
  const int needs = fp2_needs(op);
  k_fp2_elem<<<1, 1, 0, (cudaStream_t)stream>>>(op, (needs & 1) ? (uint64_t *)d_c : nullptr,
                                                (needs & 2) ? (const uint64_t *)d_a : nullptr,
                                                (needs & 4) ? (const uint64_t *)d_b : nullptr, arg,
                                                (needs & 8) ? d_flag : nullptr);
  return launched("k_fp2_elem");
}

int gm_g1_point_elem(gm_stream_t stream, uint32_t gpu_index, int op, G1Point *d_r, const G1Point *d_p,
                     const G1Point *d_q, const uint64_t *d_scalar, int scalar_limbs, uint64_t scalar_u64) {
  return point_elem<F1>(stream, gpu_index, op, d_r, d_p, d_q, d_scalar, scalar_limbs, scalar_u64);
}

int gm_g2_point_elem(gm_stream_t stream, uint32_t gpu_index, int op, G2Point *d_r, const G2Point *d_p,
                     const G2Point *d_q, const uint64_t *d_scalar, int scalar_limbs, uint64_t scalar_u64) {
  return point_elem<F2>(stream, gpu_index, op, d_r, d_p, d_q, d_scalar, scalar_limbs, scalar_u64);
}

int gm_g1_on_curve_batch(gm_stream_t stream, uint32_t gpu_index, const G1Point *d_points, int64_t n, uint8_t *d_ok) {
  if (n < 0 || (n > 0 && (!d_points || !d_ok))) return bad_arg("on_curve: bad size or null pointer");
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_on_curve<F1><<<blocks, 256, 0, (cudaStream_t)stream>>>((const uint64_t *)d_points, n, d_ok);
  return launched("k_on_curve");
}

int gm_g2_on_curve_batch(gm_stream_t stream, uint32_t gpu_index, const G2Point *d_points, int64_t n, uint8_t *d_ok) {
  if (n < 0 || (n > 0 && (!d_points || !d_ok))) return bad_arg("on_curve: bad size or null pointer");
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
  k_on_curve<F2><<<blocks, 256, 0, (cudaStream_t)stream>>>((const uint64_t *)d_points, n, d_ok);
  return launched("k_on_curve");
}

}  // extern "C"
