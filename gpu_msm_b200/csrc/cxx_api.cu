// The reference's C++ API for the MSM path (gpu_msm_b200_cxx.h), forwarding
// to the C-ABI entry points of this library.  Errors abort with a message,
// as the reference's PANIC_IF_FALSE / check_cuda_error do
// (pdroalves/gpu_msm include/device.h:11-39).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#define GM_CXX_API_IMPL  // the C-linkage init_device_generators is not declared here
#include "../../include/gpu_msm_b200.h"
#include "../../include/gpu_msm_b200_cxx.h"

namespace {

[[noreturn]] void panic(const char *where, const char *what) {
  const char *detail = gm_last_error();
  fprintf(stderr, "gpu_msm_b200: %s: %s%s%s\n", where, what, detail && *detail ? ": " : "", detail ? detail : "");
  abort();
}

void check(int rc, const char *where) {
  if (rc != 0) panic(where, "failed");
}

void check_cuda(cudaError_t e, const char *where) {
  if (e != cudaSuccess) panic(where, cudaGetErrorString(e));
}

void set_device(uint32_t gpu_index, const char *where) { check_cuda(cudaSetDevice((int)gpu_index), where); }

void sync(cudaStream_t stream, const char *where) { check_cuda(cudaStreamSynchronize(stream), where); }

// Point-type traits: group, scalar-array entry points.
template <class P>
struct Group;
template <>
struct Group<G1Point> {
  static int msm_affine(cudaStream_t s, uint32_t g, G1Point *r, const G1Point *p, const uint64_t *k, int l, int n) {
    return gm_g1_msm_device_affine(s, g, r, p, k, l, n);
  }
  static int to_mont(cudaStream_t s, uint32_t g, G1Point *p, int n) { return gm_g1_to_montgomery_batch(s, g, p, n); }
};
template <>
struct Group<G2Point> {
  static int msm_affine(cudaStream_t s, uint32_t g, G2Point *r, const G2Point *p, const uint64_t *k, int l, int n) {
    return gm_g2_msm_device_affine(s, g, r, p, k, l, n);
  }
  static int to_mont(cudaStream_t s, uint32_t g, G2Point *p, int n) { return gm_g2_to_montgomery_batch(s, g, p, n); }
};

// Host-pointer form of an element-wise device operation: copy in, run,
// copy out, synchronise (include/fp_kernels.h:15-23).
template <class E, class Op>
void host_array(cudaStream_t stream, uint32_t gpu_index, E *c, const E *a, const E *b, int n, Op op,
                const char *where) {
  if (n < 0) panic(where, "invalid size");
  if (n == 0) return;
  if (c == nullptr || a == nullptr || b == nullptr) panic(where, "null pointer argument");
  set_device(gpu_index, where);
  const size_t bytes = (size_t)n * sizeof(E);
  E *d = nullptr;
  check_cuda(cudaMallocAsync((void **)&d, 3 * bytes, stream), where);
  check_cuda(cudaMemcpyAsync(d, a, bytes, cudaMemcpyHostToDevice, stream), where);
  check_cuda(cudaMemcpyAsync(d + n, b, bytes, cudaMemcpyHostToDevice, stream), where);
  check(op(stream, gpu_index, d + 2 * (size_t)n, d, d + n, (int64_t)n), where);
  check_cuda(cudaMemcpyAsync(c, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost, stream), where);
  check_cuda(cudaFreeAsync(d, stream), where);
  sync(stream, where);
}

}  // namespace

void init_device_generators(cudaStream_t stream, uint32_t gpu_index) {
  (void)stream;
  set_device(gpu_index, "init_device_generators");
}

// ---- MSM, u64 scalars (src/curve.cu:2538-2758) ------------------------------
void point_msm_u64_async_g1(cudaStream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result,
                            const G1Point *d_points, const uint64_t *d_scalars, G1ProjectivePoint *d_scratch, int n) {
  const char *where = "point_msm_u64_async_g1";
  if (n == 0) {
    set_device(gpu_index, where);
    check_cuda(cudaMemsetAsync(d_result, 0, sizeof(G1ProjectivePoint), stream), where);
    return;
  }
  if (n < 0) panic(where, "invalid size");
  if (!d_result || !d_points || !d_scalars || !d_scratch) panic(where, "null pointer argument");
  check(gm_g1_msm_device(stream, gpu_index, d_result, d_points, d_scalars, 1, n), where);
}

void point_msm_u64_g1(cudaStream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                      const uint64_t *d_scalars, G1ProjectivePoint *d_scratch, int n) {
  point_msm_u64_async_g1(stream, gpu_index, d_result, d_points, d_scalars, d_scratch, n);
  sync(stream, "point_msm_u64_g1");
}

void point_msm_u64_async_g2(cudaStream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result,
                            const G2Point *d_points, const uint64_t *d_scalars, G2ProjectivePoint *d_scratch, int n) {
  const char *where = "point_msm_u64_async_g2";
  if (n == 0) {
    set_device(gpu_index, where);
    check_cuda(cudaMemsetAsync(d_result, 0, sizeof(G2ProjectivePoint), stream), where);
    return;
  }
  if (n < 0) panic(where, "invalid size");
  if (!d_result || !d_points || !d_scalars || !d_scratch) panic(where, "null pointer argument");
  check(gm_g2_msm_device(stream, gpu_index, d_result, d_points, d_scalars, 1, n), where);
}

void point_msm_u64_g2(cudaStream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                      const uint64_t *d_scalars, G2ProjectivePoint *d_scratch, int n) {
  point_msm_u64_async_g2(stream, gpu_index, d_result, d_points, d_scalars, d_scratch, n);
  sync(stream, "point_msm_u64_g2");
}

// ---- point at infinity, batched Montgomery conversion ------------------------
template <typename PointType>
void point_at_infinity_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result) {
  const char *where = "point_at_infinity_async";
  if (d_result == nullptr) panic(where, "null pointer argument");
  set_device(gpu_index, where);
  // coordinates zero, infinity flag set (g1/g2_point_at_infinity, src/curve.cu)
  check_cuda(cudaMemsetAsync(d_result, 0, sizeof(PointType), stream), where);
  check_cuda(cudaMemsetAsync(reinterpret_cast<char *>(d_result) + offsetof(PointType, infinity), 1, 1, stream),
             where);
}

template <typename PointType>
void point_at_infinity(cudaStream_t stream, uint32_t gpu_index, PointType *d_result) {
  point_at_infinity_async<PointType>(stream, gpu_index, d_result);
  sync(stream, "point_at_infinity");
}

template <typename PointType>
void point_to_montgomery_batch_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_points, int n) {
  const char *where = "point_to_montgomery_batch_async";
  if (n < 0 || (n > 0 && d_points == nullptr)) panic(where, "invalid argument");
  check(Group<PointType>::to_mont(stream, gpu_index, d_points, n), where);
}

template <typename PointType>
void point_to_montgomery_batch(cudaStream_t stream, uint32_t gpu_index, PointType *d_points, int n) {
  point_to_montgomery_batch_async<PointType>(stream, gpu_index, d_points, n);
  sync(stream, "point_to_montgomery_batch");
}

// ---- MSM, multi-limb scalars, affine result (src/curve.cu:2763-2826) --------
template <typename PointType>
void point_msm_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, PointType *d_scratch, int n) {
  const char *where = "point_msm_async";
  if (n == 0) {
    point_at_infinity_async<PointType>(stream, gpu_index, d_result);
    return;
  }
  if (n < 0) panic(where, "invalid size");
  if (!d_result || !d_points || !d_scalars || !d_scratch) panic(where, "null pointer argument");
  check(Group<PointType>::msm_affine(stream, gpu_index, d_result, d_points, d_scalars, scalar_limbs, n), where);
}

template <typename PointType>
void point_msm(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_points,
               const uint64_t *d_scalars, int scalar_limbs, PointType *d_scratch, int n) {
  point_msm_async<PointType>(stream, gpu_index, d_result, d_points, d_scalars, scalar_limbs, d_scratch, n);
  sync(stream, "point_msm");
}

template void point_msm_async<G1Point>(cudaStream_t, uint32_t, G1Point *, const G1Point *, const uint64_t *, int,
                                       G1Point *, int);
template void point_msm<G1Point>(cudaStream_t, uint32_t, G1Point *, const G1Point *, const uint64_t *, int, G1Point *,
                                 int);
template void point_msm_async<G2Point>(cudaStream_t, uint32_t, G2Point *, const G2Point *, const uint64_t *, int,
                                       G2Point *, int);
template void point_msm<G2Point>(cudaStream_t, uint32_t, G2Point *, const G2Point *, const uint64_t *, int, G2Point *,
                                 int);
template void point_to_montgomery_batch_async<G1Point>(cudaStream_t, uint32_t, G1Point *, int);
template void point_to_montgomery_batch<G1Point>(cudaStream_t, uint32_t, G1Point *, int);
template void point_to_montgomery_batch_async<G2Point>(cudaStream_t, uint32_t, G2Point *, int);
template void point_to_montgomery_batch<G2Point>(cudaStream_t, uint32_t, G2Point *, int);
template void point_at_infinity_async<G1Point>(cudaStream_t, uint32_t, G1Point *);
template void point_at_infinity<G1Point>(cudaStream_t, uint32_t, G1Point *);
template void point_at_infinity_async<G2Point>(cudaStream_t, uint32_t, G2Point *);
template void point_at_infinity<G2Point>(cudaStream_t, uint32_t, G2Point *);

// ---- field arrays (src/fp_kernels.cu:223, src/fp2_kernels.cu) ----------------
void fp_add_array_device(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int n) {
  const char *where = "fp_add_array_device";
  if (n < 0) panic(where, "invalid size");
  if (n == 0) return;
  if (!d_c || !d_a || !d_b) panic(where, "null pointer argument");
  check(gm_fp_add_array(stream, gpu_index, d_c, d_a, d_b, n), where);
}

void fp_mul_array_device(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int n) {
  const char *where = "fp_mul_array_device";
  if (n < 0) panic(where, "invalid size");
  if (n == 0) return;
  if (!d_c || !d_a || !d_b) panic(where, "null pointer argument");
  check(gm_fp_mul_array(stream, gpu_index, d_c, d_a, d_b, n), where);
}

void fp_add_array_host(cudaStream_t stream, uint32_t gpu_index, Fp *c, const Fp *a, const Fp *b, int n) {
  host_array(stream, gpu_index, c, a, b, n, gm_fp_add_array, "fp_add_array_host");
}

void fp_mul_array_host(cudaStream_t stream, uint32_t gpu_index, Fp *c, const Fp *a, const Fp *b, int n) {
  host_array(stream, gpu_index, c, a, b, n, gm_fp_mul_array, "fp_mul_array_host");
}

void fp2_add_array_host(cudaStream_t stream, uint32_t gpu_index, Fp2 *c, const Fp2 *a, const Fp2 *b, int n) {
  host_array(stream, gpu_index, c, a, b, n, gm_fp2_add_array, "fp2_add_array_host");
}

void fp2_mul_array_host(cudaStream_t stream, uint32_t gpu_index, Fp2 *c, const Fp2 *a, const Fp2 *b, int n) {
  host_array(stream, gpu_index, c, a, b, n, gm_fp2_mul_array, "fp2_mul_array_host");
}
