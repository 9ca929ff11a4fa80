// Test driver for the reference-compatible C++ API (gpu_msm_b200_cxx.h):
// reads inputs written by tests/test_gpu_cxx_api.py, calls the C++ entry
// points exactly as a caller of the reference's curve.h / fp_kernels.h /
// fp2_kernels.h would, and writes the outputs for comparison with the oracle.
//
//   cxx_api_driver <dir>   reads <dir>/in_*.bin, writes <dir>/out_*.bin
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/gpu_msm_b200_cxx.h"

static std::string g_dir;

template <class T>
static std::vector<T> load(const char *name) {
  std::string path = g_dir + "/" + name;
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path.c_str());
    exit(2);
  }
  fseek(f, 0, SEEK_END);
  const long bytes = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<T> v(bytes / sizeof(T));
  if (fread(v.data(), sizeof(T), v.size(), f) != v.size()) exit(2);
  fclose(f);
  return v;
}

template <class T>
static void save(const char *name, const T *p, size_t count) {
  std::string path = g_dir + "/" + name;
  FILE *f = fopen(path.c_str(), "wb");
  if (!f || fwrite(p, sizeof(T), count, f) != count) exit(3);
  fclose(f);
}

template <class T>
static T *to_device(const std::vector<T> &h) {
  T *d = nullptr;
  if (cudaMalloc(&d, (h.empty() ? 1 : h.size()) * sizeof(T)) != cudaSuccess) exit(4);
  if (!h.empty() && cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) exit(4);
  return d;
}

template <class T>
static void from_device(T *h, const T *d, size_t count) {
  if (cudaMemcpy(h, d, count * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) exit(5);
}

template <class Aff, class Prj>
static void run_group(cudaStream_t s, const char *tag, void (*msm_u64)(cudaStream_t, uint32_t, Prj *, const Aff *,
                                                                        const uint64_t *, Prj *, int)) {
  char name[64];
  snprintf(name, sizeof(name), "in_%s_points.bin", tag);
  auto pts = load<Aff>(name);
  snprintf(name, sizeof(name), "in_%s_scalars_u64.bin", tag);
  auto k64 = load<uint64_t>(name);
  snprintf(name, sizeof(name), "in_%s_scalars_5.bin", tag);
  auto k5 = load<uint64_t>(name);
  const int n = (int)pts.size();
  Aff *d_pts = to_device(pts);
  uint64_t *d_k64 = to_device(k64), *d_k5 = to_device(k5);
  Prj *d_prj, *d_scratch;
  Aff *d_aff;
  cudaMalloc(&d_prj, 2 * sizeof(Prj));
  cudaMalloc(&d_scratch, sizeof(Prj));
  cudaMalloc(&d_aff, 2 * sizeof(Aff));
  // u64 scalars, projective result; then n == 0 (identity)
  msm_u64(s, 0, d_prj, d_pts, d_k64, d_scratch, n);
  msm_u64(s, 0, d_prj + 1, d_pts, d_k64, d_scratch, 0);
  cudaStreamSynchronize(s);
  // five-limb scalars, affine result; then n == 0
  point_msm<Aff>(s, 0, d_aff, d_pts, d_k5, 5, reinterpret_cast<Aff *>(d_scratch), n);
  point_msm_async<Aff>(s, 0, d_aff + 1, d_pts, d_k5, 5, reinterpret_cast<Aff *>(d_scratch), 0);
  cudaStreamSynchronize(s);
  Prj prj[2];
  Aff aff[2];
  from_device(prj, d_prj, 2);
  from_device(aff, d_aff, 2);
  snprintf(name, sizeof(name), "out_%s_msm_u64.bin", tag);
  save(name, prj, 2);
  snprintf(name, sizeof(name), "out_%s_msm_affine.bin", tag);
  save(name, aff, 2);
  // standard -> Montgomery in place
  snprintf(name, sizeof(name), "in_%s_points_std.bin", tag);
  auto std_pts = load<Aff>(name);
  Aff *d_std = to_device(std_pts);
  point_to_montgomery_batch<Aff>(s, 0, d_std, (int)std_pts.size());
  std::vector<Aff> conv(std_pts.size());
  from_device(conv.data(), d_std, conv.size());
  snprintf(name, sizeof(name), "out_%s_to_mont.bin", tag);
  save(name, conv.data(), conv.size());
  cudaFree(d_pts);
  cudaFree(d_k64);
  cudaFree(d_k5);
  cudaFree(d_prj);
  cudaFree(d_scratch);
  cudaFree(d_aff);
  cudaFree(d_std);
}

// Single-element stream APIs and host-pointer helpers: one call of each on
// the first inputs, results in a fixed order (out_elem_*.bin).
template <class E>
static E run_dev(cudaStream_t s, void (*op)(cudaStream_t, uint32_t, E *, const E *, const E *), const E &a,
                 const E &b) {
  std::vector<E> in{a, b, E{}};
  E *d = to_device(in);
  op(s, 0, d + 2, d, d + 1);
  cudaStreamSynchronize(s);
  E r;
  from_device(&r, d + 2, 1);
  cudaFree(d);
  return r;
}
template <class E>
static E run_dev(cudaStream_t s, void (*op)(cudaStream_t, uint32_t, E *, const E *), const E &a) {
  std::vector<E> in{a, E{}};
  E *d = to_device(in);
  op(s, 0, d + 1, d);
  cudaStreamSynchronize(s);
  E r;
  from_device(&r, d + 1, 1);
  cudaFree(d);
  return r;
}

static void run_elements(cudaStream_t s, const Fp &a, const Fp &b, const Fp2 &a2, const Fp2 &b2) {
  std::vector<Fp> f;
  std::vector<int32_t> flags;
  f.push_back(run_dev<Fp>(s, fp_add, a, b));
  f.push_back(run_dev<Fp>(s, fp_sub_async, a, b));
  f.push_back(run_dev<Fp>(s, fp_mul, a, b));
  f.push_back(run_dev<Fp>(s, fp_div_async, a, b));
  f.push_back(run_dev<Fp>(s, fp_mont_mul, a, b));
  f.push_back(run_dev<Fp>(s, fp_neg_async, a));
  f.push_back(run_dev<Fp>(s, fp_inv, a));
  f.push_back(run_dev<Fp>(s, fp_to_montgomery_async, a));
  f.push_back(run_dev<Fp>(s, fp_from_montgomery, a));
  f.push_back(run_dev<Fp>(s, fp_copy_async, a));
  {
    std::vector<Fp> z(2);
    Fp *d = to_device(z);
    fp_zero(s, 0, d);
    fp_one_async(s, 0, d + 1);
    cudaStreamSynchronize(s);
    from_device(z.data(), d, 2);
    cudaFree(d);
    f.insert(f.end(), z.begin(), z.end());
  }
  Fp r;
  fp_add_gpu(s, 0, &r, &a, &b);
  f.push_back(r);
  fp_sub_gpu(s, 0, &r, &a, &b);
  f.push_back(r);
  fp_mul_gpu(s, 0, &r, &a, &b);
  f.push_back(r);
  fp_neg_gpu(s, 0, &r, &a);
  f.push_back(r);
  fp_inv_gpu(s, 0, &r, &a);
  f.push_back(r);
  fp_div_gpu(s, 0, &r, &a, &b);
  f.push_back(r);
  fp_to_montgomery_gpu(s, 0, &r, &a);
  f.push_back(r);
  fp_from_montgomery_gpu(s, 0, &r, &a);
  f.push_back(r);
  fp_mont_mul_gpu(s, 0, &r, &a, &b);
  f.push_back(r);
  fp_copy_gpu(s, 0, &r, &a);
  f.push_back(r);
  r = b;
  fp_cmov_gpu(s, 0, &r, &a, 1);
  f.push_back(r);
  r = b;
  fp_cmov_gpu(s, 0, &r, &a, 0);
  f.push_back(r);
  fp_pow_u64_gpu(s, 0, &r, &a, 65537);
  f.push_back(r);
  Fp sq;
  fp_mul_gpu(s, 0, &sq, &a, &a);
  flags.push_back(fp_sqrt_gpu(s, 0, &r, &sq));
  f.push_back(r);
  flags.push_back(fp_cmp_gpu(s, 0, &a, &b));
  flags.push_back(fp_is_zero_gpu(s, 0, &a));
  Fp one{};
  one.limb[0] = 1;
  flags.push_back(fp_is_one_gpu(s, 0, &one));
  flags.push_back(fp_is_quadratic_residue_gpu(s, 0, &a));
  save("out_elem_fp.bin", f.data(), f.size());

  std::vector<Fp2> g;
  g.push_back(run_dev<Fp2>(s, fp2_add, a2, b2));
  g.push_back(run_dev<Fp2>(s, fp2_sub_async, a2, b2));
  g.push_back(run_dev<Fp2>(s, fp2_mul, a2, b2));
  g.push_back(run_dev<Fp2>(s, fp2_div_async, a2, b2));
  g.push_back(run_dev<Fp2>(s, fp2_square, a2));
  g.push_back(run_dev<Fp2>(s, fp2_neg_async, a2));
  g.push_back(run_dev<Fp2>(s, fp2_conjugate, a2));
  g.push_back(run_dev<Fp2>(s, fp2_inv_async, a2));
  g.push_back(run_dev<Fp2>(s, fp2_copy, a2));
  Fp2 r2;
  fp2_add_gpu(&r2, &a2, &b2);
  g.push_back(r2);
  fp2_sub_gpu(&r2, &a2, &b2);
  g.push_back(r2);
  fp2_mul_gpu(&r2, &a2, &b2);
  g.push_back(r2);
  fp2_neg_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_conjugate_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_square_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_inv_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_div_gpu(&r2, &a2, &b2);
  g.push_back(r2);
  fp2_mul_by_i_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_frobenius_gpu(&r2, &a2);
  g.push_back(r2);
  fp2_copy_gpu(&r2, &a2);
  g.push_back(r2);
  r2 = b2;
  fp2_cmov_gpu(&r2, &a2, 1);
  g.push_back(r2);
  flags.push_back(fp2_cmp_gpu(&a2, &b2));
  flags.push_back(fp2_is_zero_gpu(&a2));
  flags.push_back(fp2_is_one_gpu(&a2));
  save("out_elem_fp2.bin", g.data(), g.size());
  save("out_elem_flags.bin", flags.data(), flags.size());
}

template <class Aff>
static void run_point_elements(cudaStream_t s, const char *tag) {
  char name[64];
  snprintf(name, sizeof(name), "in_%s_points.bin", tag);
  auto pts = load<Aff>(name);
  snprintf(name, sizeof(name), "in_%s_scalars_u64.bin", tag);
  auto k64 = load<uint64_t>(name);
  snprintf(name, sizeof(name), "in_%s_scalars_5.bin", tag);
  auto k5 = load<uint64_t>(name);
  snprintf(name, sizeof(name), "in_%s_points_std.bin", tag);
  auto std_pts = load<Aff>(name);
  std::vector<Aff> in{pts[0], pts[1], std_pts[0]};
  Aff *d = to_device(in), *r;
  uint64_t *dk = to_device(std::vector<uint64_t>(k5.begin(), k5.begin() + 5));
  cudaMalloc(&r, 7 * sizeof(Aff));
  point_add<Aff>(s, 0, r, d, d + 1);
  point_double_async<Aff>(s, 0, r + 1, d);
  point_neg<Aff>(s, 0, r + 2, d);
  point_scalar_mul_u64_async<Aff>(s, 0, r + 3, d, k64[0]);
  point_scalar_mul<Aff>(s, 0, r + 4, d, dk, 5);
  point_to_montgomery_async<Aff>(s, 0, r + 5, d + 2);
  point_from_montgomery<Aff>(s, 0, r + 6, d);
  std::vector<Aff> out(7);
  from_device(out.data(), r, 7);
  snprintf(name, sizeof(name), "out_elem_%s.bin", tag);
  save(name, out.data(), out.size());
  cudaFree(d);
  cudaFree(dk);
  cudaFree(r);
}

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s <dir>\n", argv[0]);
    return 1;
  }
  g_dir = argv[1];
  cudaStream_t s;
  if (cudaStreamCreate(&s) != cudaSuccess) return 4;
  init_device_generators(s, 0);
  run_group<G1Point, G1ProjectivePoint>(s, "g1", point_msm_u64_g1);
  run_group<G2Point, G2ProjectivePoint>(s, "g2", point_msm_u64_g2);

  auto a = load<Fp>("in_fp_a.bin"), b = load<Fp>("in_fp_b.bin");
  const int m = (int)a.size();
  std::vector<Fp> c(m);
  fp_mul_array_host(s, 0, c.data(), a.data(), b.data(), m);
  save("out_fp_mul_host.bin", c.data(), c.size());
  fp_add_array_host(s, 0, c.data(), a.data(), b.data(), m);
  save("out_fp_add_host.bin", c.data(), c.size());
  Fp *d_a = to_device(a), *d_b = to_device(b), *d_c = to_device(c);
  fp_mul_array_device(s, 0, d_c, d_a, d_b, m);
  cudaStreamSynchronize(s);
  from_device(c.data(), d_c, c.size());
  save("out_fp_mul_device.bin", c.data(), c.size());
  fp_add_array_device(s, 0, d_c, d_a, d_b, m);
  cudaStreamSynchronize(s);
  from_device(c.data(), d_c, c.size());
  save("out_fp_add_device.bin", c.data(), c.size());

  auto a2 = load<Fp2>("in_fp2_a.bin"), b2 = load<Fp2>("in_fp2_b.bin");
  std::vector<Fp2> c2(a2.size());
  fp2_mul_array_host(s, 0, c2.data(), a2.data(), b2.data(), (int)a2.size());
  save("out_fp2_mul_host.bin", c2.data(), c2.size());
  fp2_add_array_host(s, 0, c2.data(), a2.data(), b2.data(), (int)a2.size());
  save("out_fp2_add_host.bin", c2.data(), c2.size());

  run_elements(s, a[0], b[0], a2[0], b2[0]);
  run_point_elements<G1Point>(s, "g1");
  run_point_elements<G2Point>(s, "g2");
  cudaStreamDestroy(s);
  printf("cxx_api_driver: ok\n");
  return 0;
}
