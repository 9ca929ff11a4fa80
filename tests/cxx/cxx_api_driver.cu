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
  cudaStreamDestroy(s);
  printf("cxx_api_driver: ok\n");
  return 0;
}
