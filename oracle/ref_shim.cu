// Builds the reference's own host code (pdroalves/gpu_msm src/fp.cu,
// src/fp2.cu, src/device.cu, src/curve.cu, compiled by oracle/Makefile from
// where they lie in the reference tree; nothing is copied) and exposes a few of its host functions
// through extern "C" so Python tests can pin the oracle restatement against
// it.  TEST INFRASTRUCTURE ONLY: the output goes to oracle/_ref/ and is used
// by tests/ and by bench.py's CPU-baseline leg, never by the product path.
//
// The reference has no host-side MSM entry point (its MSM launches kernels),
// so ref_g{1,2}_msm_pippenger arranges the reference's host functions the way
// its MSM driver does (src/curve.cu:2538-2677): 4-bit unsigned windows,
// projective buckets filled with affine_to_projective + projective_point_add,
// and combine_buckets_cpu_projective_g1/_g2 per window, MSB first.  Windows
// are accumulated in parallel by std::thread; the combine is serial.
#include "src/curve.cu"

#include <string>
#include <thread>
#include <vector>

// point_to/from_montgomery are kernels in the reference
// (src/curve.cu:2313-2340); their host-function bodies, through the same traits
template <class P>
void ref_point_convert(P &r, const P &p, bool to) {
  using Tr = PointTraits<P>;
  if (p.infinity) {
    r.infinity = true;
    Tr::field_zero(r.x);
    Tr::field_zero(r.y);
  } else if (to) {
    Tr::field_to_montgomery(r.x, p.x);
    Tr::field_to_montgomery(r.y, p.y);
    r.infinity = false;
  } else {
    Tr::field_from_montgomery(r.x, p.x);
    Tr::field_from_montgomery(r.y, p.y);
    r.infinity = false;
  }
}

template <class P>
int ref_point_elem(const char *op, P *r, const P *p, const P *q, const uint64_t *k, int limbs, uint64_t k64) {
  const std::string o(op);
  if (o == "add") point_add(*r, *p, *q);
  else if (o == "double") point_double(*r, *p);
  else if (o == "neg") point_neg(*r, *p);
  else if (o == "scalar_mul") point_scalar_mul(*r, *p, k, limbs);
  else if (o == "scalar_mul_u64") point_scalar_mul(*r, *p, &k64, 1);
  else if (o == "to_mont") ref_point_convert(*r, *p, true);
  else if (o == "from_mont") ref_point_convert(*r, *p, false);
  else if (o == "at_infinity") PointTraits<P>::point_at_infinity(*r);
  else return -99;
  return 0;
}
extern "C" {

void ref_fp_mont_mul_batch(Fp *c, const Fp *a, const Fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_mont_mul(c[i], a[i], b[i]);
}
void ref_fp_mul_batch(Fp *c, const Fp *a, const Fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_mul(c[i], a[i], b[i]);
}
void ref_fp_add_batch(Fp *c, const Fp *a, const Fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_add(c[i], a[i], b[i]);
}
void ref_fp_sub_batch(Fp *c, const Fp *a, const Fp *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_sub(c[i], a[i], b[i]);
}
void ref_fp_to_mont_batch(Fp *c, const Fp *a, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_to_montgomery(c[i], a[i]);
}
void ref_fp_from_mont_batch(Fp *c, const Fp *a, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp_from_montgomery(c[i], a[i]);
}
void ref_fp_mont_inv(Fp *c, const Fp *a) { fp_mont_inv(*c, *a); }
void ref_fp2_mont_mul_batch(Fp2 *c, const Fp2 *a, const Fp2 *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp2_mont_mul(c[i], a[i], b[i]);
}
void ref_fp2_mul_batch(Fp2 *c, const Fp2 *a, const Fp2 *b, int64_t n) {
  for (int64_t i = 0; i < n; i++) fp2_mul(c[i], a[i], b[i]);
}
void ref_fp2_mont_inv(Fp2 *c, const Fp2 *a) { fp2_mont_inv(*c, *a); }

void ref_g1_add(G1Point *r, const G1Point *a, const G1Point *b) { point_add(*r, *a, *b); }
void ref_g2_add(G2Point *r, const G2Point *a, const G2Point *b) { point_add(*r, *a, *b); }
void ref_g1_double(G1Point *r, const G1Point *a) { point_double(*r, *a); }
void ref_g2_double(G2Point *r, const G2Point *a) { point_double(*r, *a); }
void ref_g1_scalar_mul(G1Point *r, const G1Point *p, const uint64_t *k, int limbs) {
  point_scalar_mul(*r, *p, k, limbs);
}
void ref_g2_scalar_mul(G2Point *r, const G2Point *p, const uint64_t *k, int limbs) {
  point_scalar_mul(*r, *p, k, limbs);
}
void ref_g1p_add(G1ProjectivePoint *r, const G1ProjectivePoint *a, const G1ProjectivePoint *b) {
  projective_point_add(*r, *a, *b);
}
void ref_g1p_double(G1ProjectivePoint *r, const G1ProjectivePoint *a) {
  projective_point_double(*r, *a);
}
void ref_g2p_add(G2ProjectivePoint *r, const G2ProjectivePoint *a, const G2ProjectivePoint *b) {
  projective_point_add(*r, *a, *b);
}
void ref_g2p_double(G2ProjectivePoint *r, const G2ProjectivePoint *a) {
  projective_point_double(*r, *a);
}
void ref_g1_proj_to_affine(G1Point *r, const G1ProjectivePoint *p) { projective_to_affine_g1(*r, *p); }
void ref_g2_proj_to_affine(G2Point *r, const G2ProjectivePoint *p) { projective_to_affine_g2(*r, *p); }

// Projective result of the reference-structured CPU Pippenger, then
// projective_to_affine (Montgomery form), like the reference tests do.
void ref_g1_msm_pippenger(G1Point *r, G1ProjectivePoint *r_proj, const G1Point *pts,
                          const uint64_t *scalars, int limbs, int64_t n, int threads) {
  const int nw = limbs * 64 / MSM_WINDOW_SIZE;
  int th = threads < 1 ? 1 : (threads > nw ? nw : threads);
  std::vector<G1ProjectivePoint> buckets((size_t)nw * MSM_BUCKET_COUNT);
  auto work = [&](int w0, int w1) {
    for (int w = w0; w < w1; w++) {
      G1ProjectivePoint *b = &buckets[(size_t)w * MSM_BUCKET_COUNT];
      for (int j = 0; j < MSM_BUCKET_COUNT; j++) g1_projective_point_at_infinity(b[j]);
      const int limb = (w * MSM_WINDOW_SIZE) / 64, shift = (w * MSM_WINDOW_SIZE) % 64;
      for (int64_t i = 0; i < n; i++) {
        const int d = (int)((scalars[i * limbs + limb] >> shift) & (MSM_BUCKET_COUNT - 1));
        if (d == 0 || pts[i].infinity) continue;
        G1ProjectivePoint pp, t;
        affine_to_projective(pp, pts[i]);
        projective_point_add(t, b[d], pp);
        b[d] = t;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < th; t++)
    pool.emplace_back(work, (int)((int64_t)nw * t / th), (int)((int64_t)nw * (t + 1) / th));
  for (auto &x : pool) x.join();
  G1ProjectivePoint res;
  g1_projective_point_at_infinity(res);
  for (int w = nw - 1; w >= 0; w--)
    combine_buckets_cpu_projective_g1(res, &buckets[(size_t)w * MSM_BUCKET_COUNT], MSM_BUCKET_COUNT, w);
  if (r_proj) *r_proj = res;
  projective_to_affine_g1(*r, res);
}

void ref_g2_msm_pippenger(G2Point *r, G2ProjectivePoint *r_proj, const G2Point *pts,
                          const uint64_t *scalars, int limbs, int64_t n, int threads) {
  const int nw = limbs * 64 / MSM_WINDOW_SIZE;
  int th = threads < 1 ? 1 : (threads > nw ? nw : threads);
  std::vector<G2ProjectivePoint> buckets((size_t)nw * MSM_BUCKET_COUNT);
  auto work = [&](int w0, int w1) {
    for (int w = w0; w < w1; w++) {
      G2ProjectivePoint *b = &buckets[(size_t)w * MSM_BUCKET_COUNT];
      for (int j = 0; j < MSM_BUCKET_COUNT; j++) g2_projective_point_at_infinity(b[j]);
      const int limb = (w * MSM_WINDOW_SIZE) / 64, shift = (w * MSM_WINDOW_SIZE) % 64;
      for (int64_t i = 0; i < n; i++) {
        const int d = (int)((scalars[i * limbs + limb] >> shift) & (MSM_BUCKET_COUNT - 1));
        if (d == 0 || pts[i].infinity) continue;
        G2ProjectivePoint pp, t;
        affine_to_projective(pp, pts[i]);
        projective_point_add(t, b[d], pp);
        b[d] = t;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < th; t++)
    pool.emplace_back(work, (int)((int64_t)nw * t / th), (int)((int64_t)nw * (t + 1) / th));
  for (auto &x : pool) x.join();
  G2ProjectivePoint res;
  g2_projective_point_at_infinity(res);
  for (int w = nw - 1; w >= 0; w--)
    combine_buckets_cpu_projective_g2(res, &buckets[(size_t)w * MSM_BUCKET_COUNT], MSM_BUCKET_COUNT, w);
  if (r_proj) *r_proj = res;
  projective_to_affine_g2(*r, res);
}

// Single-element operations by name: the reference's __host__ __device__
// functions that its stream-API kernels call (src/fp_kernels.cu:57-148,
// src/fp2_kernels.cu:40-110, src/curve.cu:2288-2380).  Returns the value of
// the predicates (cmp, is_zero, is_one, is_qr, sqrt), else 0; -99 for an
// unknown name.
int ref_fp_elem(const char *op, Fp *c, const Fp *a, const Fp *b, uint64_t arg) {
  const std::string o(op);
  if (o == "add") fp_add(*c, *a, *b);
  else if (o == "sub") fp_sub(*c, *a, *b);
  else if (o == "mul") fp_mul(*c, *a, *b);
  else if (o == "neg") fp_neg(*c, *a);
  else if (o == "inv") fp_inv(*c, *a);
  else if (o == "div") fp_div(*c, *a, *b);
  else if (o == "copy") fp_copy(*c, *a);
  else if (o == "zero") fp_zero(*c);
  else if (o == "one") fp_one(*c);
  else if (o == "to_mont") fp_to_montgomery(*c, *a);
  else if (o == "from_mont") fp_from_montgomery(*c, *a);
  else if (o == "mont_mul") fp_mont_mul(*c, *a, *b);
  else if (o == "cmp") return fp_cmp(*a, *b);
  else if (o == "is_zero") return fp_is_zero(*a);
  else if (o == "is_one") return fp_is_one(*a);
  else if (o == "cmov") fp_cmov(*c, *a, arg);
  else if (o == "sqrt") return fp_sqrt(*c, *a);
  else if (o == "is_qr") return fp_is_quadratic_residue(*a);
  else if (o == "pow_u64") fp_pow_u64(*c, *a, arg);
  else return -99;
  return 0;
}

int ref_fp2_elem(const char *op, Fp2 *c, const Fp2 *a, const Fp2 *b, uint64_t arg) {
  const std::string o(op);
  if (o == "add") fp2_add(*c, *a, *b);
  else if (o == "sub") fp2_sub(*c, *a, *b);
  else if (o == "mul") fp2_mul(*c, *a, *b);
  else if (o == "square") fp2_square(*c, *a);
  else if (o == "neg") fp2_neg(*c, *a);
  else if (o == "conjugate") fp2_conjugate(*c, *a);
  else if (o == "inv") fp2_inv(*c, *a);
  else if (o == "div") fp2_div(*c, *a, *b);
  else if (o == "copy") fp2_copy(*c, *a);
  else if (o == "mul_by_i") fp2_mul_by_i(*c, *a);
  else if (o == "frobenius") fp2_frobenius(*c, *a);
  else if (o == "cmp") return fp2_cmp(*a, *b);
  else if (o == "is_zero") return fp2_is_zero(*a);
  else if (o == "is_one") return fp2_is_one(*a);
  else if (o == "cmov") fp2_cmov(*c, *a, arg);
  else if (o == "mont_mul") fp2_mont_mul(*c, *a, *b);
  else return -99;
  return 0;
}

int ref_g1_point_elem(const char *op, G1Point *r, const G1Point *p, const G1Point *q, const uint64_t *k, int limbs,
                      uint64_t k64) {
  return ref_point_elem(op, r, p, q, k, limbs, k64);
}
int ref_g2_point_elem(const char *op, G2Point *r, const G2Point *p, const G2Point *q, const uint64_t *k, int limbs,
                      uint64_t k64) {
  return ref_point_elem(op, r, p, q, k, limbs, k64);
}

}  // extern "C"
