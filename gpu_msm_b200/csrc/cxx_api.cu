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

// ---- single-element stream APIs on device pointers -------------------------
// include/fp.h:158-204 and include/fp2.h:99-133 (src/fp_kernels.cu:753-900,
// src/fp2_kernels.cu:564-680): one kernel each through gm_fp_elem /
// gm_fp2_elem; the names without _async synchronise the stream.
#define GM_SYNC_PAIR(name, params, args, call)      \
  void name##_async params { check(call, #name "_async"); } \
  void name params {                                \
    name##_async args;                              \
    sync(stream, #name);                            \
  }

#define GM_FP_BINARY(name, OP)                                                                    \
  GM_SYNC_PAIR(name, (cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b), \
               (stream, gpu_index, d_c, d_a, d_b), gm_fp_elem(stream, gpu_index, OP, d_c, d_a, d_b, 0, nullptr))
#define GM_FP_UNARY(name, OP)                                                                         \
  GM_SYNC_PAIR(name, (cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a), (stream, gpu_index, d_c, d_a), \
               gm_fp_elem(stream, gpu_index, OP, d_c, d_a, nullptr, 0, nullptr))
#define GM_FP_NULLARY(name, OP)                                                                           \
  GM_SYNC_PAIR(name, (cudaStream_t stream, uint32_t gpu_index, Fp *d_a), (stream, gpu_index, d_a), \
               gm_fp_elem(stream, gpu_index, OP, d_a, nullptr, nullptr, 0, nullptr))
#define GM_FP2_BINARY(name, OP)                                                                           \
  GM_SYNC_PAIR(name, (cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b), \
               (stream, gpu_index, d_c, d_a, d_b), gm_fp2_elem(stream, gpu_index, OP, d_c, d_a, d_b, 0, nullptr))
#define GM_FP2_UNARY(name, OP)                                                                    \
  GM_SYNC_PAIR(name, (cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a),          \
               (stream, gpu_index, d_c, d_a), gm_fp2_elem(stream, gpu_index, OP, d_c, d_a, nullptr, 0, nullptr))

GM_FP_BINARY(fp_add, GM_FP_ADD)
GM_FP_BINARY(fp_sub, GM_FP_SUB)
GM_FP_BINARY(fp_mul, GM_FP_MUL)
GM_FP_BINARY(fp_div, GM_FP_DIV)
GM_FP_BINARY(fp_mont_mul, GM_FP_MONT_MUL)
GM_FP_UNARY(fp_neg, GM_FP_NEG)
GM_FP_UNARY(fp_inv, GM_FP_INV)
GM_FP_UNARY(fp_to_montgomery, GM_FP_TO_MONT)
GM_FP_UNARY(fp_from_montgomery, GM_FP_FROM_MONT)
// fp_copy's parameters are named (d_dst, d_src) in the reference; same order
GM_FP_UNARY(fp_copy, GM_FP_COPY)
GM_FP_NULLARY(fp_zero, GM_FP_ZERO)
GM_FP_NULLARY(fp_one, GM_FP_ONE)

GM_FP2_BINARY(fp2_add, GM_FP2_ADD)
GM_FP2_BINARY(fp2_sub, GM_FP2_SUB)
GM_FP2_BINARY(fp2_mul, GM_FP2_MUL)
GM_FP2_BINARY(fp2_div, GM_FP2_DIV)
GM_FP2_UNARY(fp2_square, GM_FP2_SQUARE)
GM_FP2_UNARY(fp2_neg, GM_FP2_NEG)
GM_FP2_UNARY(fp2_conjugate, GM_FP2_CONJUGATE)
GM_FP2_UNARY(fp2_inv, GM_FP2_INV)
GM_FP2_UNARY(fp2_copy, GM_FP2_COPY)

// ---- point stream APIs (include/curve.h:156-205, src/curve.cu:2385-2500) ----
namespace {
template <class P>
struct PointElem;
template <>
struct PointElem<G1Point> {
  static int run(cudaStream_t s, uint32_t g, int op, G1Point *r, const G1Point *p, const G1Point *q,
                 const uint64_t *k, int limbs, uint64_t k64) {
    return gm_g1_point_elem(s, g, op, r, p, q, k, limbs, k64);
  }
};
template <>
struct PointElem<G2Point> {
  static int run(cudaStream_t s, uint32_t g, int op, G2Point *r, const G2Point *p, const G2Point *q,
                 const uint64_t *k, int limbs, uint64_t k64) {
    return gm_g2_point_elem(s, g, op, r, p, q, k, limbs, k64);
  }
};
}  // namespace

template <typename PointType>
void point_add_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p1,
                     const PointType *d_p2) {
  check(PointElem<PointType>::run(stream, gpu_index, GM_PT_ADD, d_result, d_p1, d_p2, nullptr, 0, 0),
        "point_add_async");
}
template <typename PointType>
void point_add(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p1,
               const PointType *d_p2) {
  point_add_async<PointType>(stream, gpu_index, d_result, d_p1, d_p2);
  sync(stream, "point_add");
}

#define GM_POINT_UNARY(name, OP)                                                                              \
  template <typename PointType>                                                                               \
  void name##_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p) {      \
    check(PointElem<PointType>::run(stream, gpu_index, OP, d_result, d_p, nullptr, nullptr, 0, 0), #name "_async"); \
  }                                                                                                           \
  template <typename PointType>                                                                               \
  void name(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p) {             \
    name##_async<PointType>(stream, gpu_index, d_result, d_p);                                                \
    sync(stream, #name);                                                                                      \
  }
GM_POINT_UNARY(point_double, GM_PT_DOUBLE)
GM_POINT_UNARY(point_neg, GM_PT_NEG)
GM_POINT_UNARY(point_to_montgomery, GM_PT_TO_MONT)
GM_POINT_UNARY(point_from_montgomery, GM_PT_FROM_MONT)

template <typename PointType>
void point_scalar_mul_u64_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result,
                                const PointType *d_point, uint64_t scalar) {
  check(PointElem<PointType>::run(stream, gpu_index, GM_PT_SCALAR_MUL_U64, d_result, d_point, nullptr, nullptr, 0,
                                  scalar),
        "point_scalar_mul_u64_async");
}
template <typename PointType>
void point_scalar_mul_u64(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                          uint64_t scalar) {
  point_scalar_mul_u64_async<PointType>(stream, gpu_index, d_result, d_point, scalar);
  sync(stream, "point_scalar_mul_u64");
}

template <typename PointType>
void point_scalar_mul_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                            const uint64_t *d_scalar, int scalar_limbs) {
  check(PointElem<PointType>::run(stream, gpu_index, GM_PT_SCALAR_MUL, d_result, d_point, nullptr, d_scalar,
                                  scalar_limbs, 0),
        "point_scalar_mul_async");
}
template <typename PointType>
void point_scalar_mul(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                      const uint64_t *d_scalar, int scalar_limbs) {
  point_scalar_mul_async<PointType>(stream, gpu_index, d_result, d_point, d_scalar, scalar_limbs);
  sync(stream, "point_scalar_mul");
}

#define GM_POINT_INSTANTIATE(P)                                                                            \
  template void point_add_async<P>(cudaStream_t, uint32_t, P *, const P *, const P *);                     \
  template void point_add<P>(cudaStream_t, uint32_t, P *, const P *, const P *);                           \
  template void point_double_async<P>(cudaStream_t, uint32_t, P *, const P *);                             \
  template void point_double<P>(cudaStream_t, uint32_t, P *, const P *);                                   \
  template void point_neg_async<P>(cudaStream_t, uint32_t, P *, const P *);                                \
  template void point_neg<P>(cudaStream_t, uint32_t, P *, const P *);                                      \
  template void point_to_montgomery_async<P>(cudaStream_t, uint32_t, P *, const P *);                      \
  template void point_to_montgomery<P>(cudaStream_t, uint32_t, P *, const P *);                            \
  template void point_from_montgomery_async<P>(cudaStream_t, uint32_t, P *, const P *);                    \
  template void point_from_montgomery<P>(cudaStream_t, uint32_t, P *, const P *);                          \
  template void point_scalar_mul_u64_async<P>(cudaStream_t, uint32_t, P *, const P *, uint64_t);           \
  template void point_scalar_mul_u64<P>(cudaStream_t, uint32_t, P *, const P *, uint64_t);                 \
  template void point_scalar_mul_async<P>(cudaStream_t, uint32_t, P *, const P *, const uint64_t *, int);  \
  template void point_scalar_mul<P>(cudaStream_t, uint32_t, P *, const P *, const uint64_t *, int);
GM_POINT_INSTANTIATE(G1Point)
GM_POINT_INSTANTIATE(G2Point)

// ---- host-pointer single-element helpers ------------------------------------
// include/fp_kernels.h:26-38 (stream and device given) and
// include/fp2_kernels.h:21-37 (current device, default stream): copy the
// operands to the device, run the element op, copy the result (and the
// flag of the predicates) back and synchronise.  For cmov `result` is read
// as well as written.
namespace {
template <class E, class Fn>
int32_t host_elem(cudaStream_t s, uint32_t g, Fn fn, int op, E *result, const E *a, const E *b, uint64_t arg,
                  bool result_in, const char *where) {
  set_device(g, where);
  struct Buf {
    E c, a, b;
    int32_t flag;
  };
  Buf *d = nullptr;
  check_cuda(cudaMallocAsync((void **)&d, sizeof(Buf), s), where);
  if (result_in) check_cuda(cudaMemcpyAsync(&d->c, result, sizeof(E), cudaMemcpyHostToDevice, s), where);
  if (a) check_cuda(cudaMemcpyAsync(&d->a, a, sizeof(E), cudaMemcpyHostToDevice, s), where);
  if (b) check_cuda(cudaMemcpyAsync(&d->b, b, sizeof(E), cudaMemcpyHostToDevice, s), where);
  check_cuda(cudaMemsetAsync(&d->flag, 0, sizeof(int32_t), s), where);
  check(fn(s, g, op, result ? &d->c : nullptr, a ? &d->a : nullptr, b ? &d->b : nullptr, arg, &d->flag), where);
  int32_t flag = 0;
  if (result) check_cuda(cudaMemcpyAsync(result, &d->c, sizeof(E), cudaMemcpyDeviceToHost, s), where);
  check_cuda(cudaMemcpyAsync(&flag, &d->flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s), where);
  check_cuda(cudaFreeAsync(d, s), where);
  sync(s, where);
  return flag;
}

int32_t fp_host(cudaStream_t s, uint32_t g, int op, Fp *r, const Fp *a, const Fp *b, uint64_t arg, const char *w,
                bool r_in = false) {
  return host_elem<Fp>(s, g, gm_fp_elem, op, r, a, b, arg, r_in, w);
}

uint32_t current_device(const char *where) {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), where);
  return (uint32_t)dev;
}

int32_t fp2_host(int op, Fp2 *r, const Fp2 *a, const Fp2 *b, uint64_t arg, const char *w, bool r_in = false) {
  return host_elem<Fp2>(nullptr, current_device(w), gm_fp2_elem, op, r, a, b, arg, r_in, w);
}
}  // namespace

void fp_add_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a, const Fp *b) {
  fp_host(s, g, GM_FP_ADD, result, a, b, 0, "fp_add_gpu");
}
void fp_sub_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a, const Fp *b) {
  fp_host(s, g, GM_FP_SUB, result, a, b, 0, "fp_sub_gpu");
}
void fp_mul_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a, const Fp *b) {
  fp_host(s, g, GM_FP_MUL, result, a, b, 0, "fp_mul_gpu");
}
void fp_neg_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  fp_host(s, g, GM_FP_NEG, result, a, nullptr, 0, "fp_neg_gpu");
}
void fp_inv_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  fp_host(s, g, GM_FP_INV, result, a, nullptr, 0, "fp_inv_gpu");
}
void fp_div_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a, const Fp *b) {
  fp_host(s, g, GM_FP_DIV, result, a, b, 0, "fp_div_gpu");
}
int fp_cmp_gpu(cudaStream_t s, uint32_t g, const Fp *a, const Fp *b) {
  return fp_host(s, g, GM_FP_CMP, nullptr, a, b, 0, "fp_cmp_gpu");
}
bool fp_is_zero_gpu(cudaStream_t s, uint32_t g, const Fp *a) {
  return fp_host(s, g, GM_FP_IS_ZERO, nullptr, a, nullptr, 0, "fp_is_zero_gpu") != 0;
}
bool fp_is_one_gpu(cudaStream_t s, uint32_t g, const Fp *a) {
  return fp_host(s, g, GM_FP_IS_ONE, nullptr, a, nullptr, 0, "fp_is_one_gpu") != 0;
}
void fp_to_montgomery_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  fp_host(s, g, GM_FP_TO_MONT, result, a, nullptr, 0, "fp_to_montgomery_gpu");
}
void fp_from_montgomery_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  fp_host(s, g, GM_FP_FROM_MONT, result, a, nullptr, 0, "fp_from_montgomery_gpu");
}
void fp_mont_mul_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a, const Fp *b) {
  fp_host(s, g, GM_FP_MONT_MUL, result, a, b, 0, "fp_mont_mul_gpu");
}
void fp_copy_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  fp_host(s, g, GM_FP_COPY, result, a, nullptr, 0, "fp_copy_gpu");
}
void fp_cmov_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *src, uint64_t condition) {
  fp_host(s, g, GM_FP_CMOV, result, src, nullptr, condition, "fp_cmov_gpu", true);
}
bool fp_sqrt_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *a) {
  return fp_host(s, g, GM_FP_SQRT, result, a, nullptr, 0, "fp_sqrt_gpu") != 0;
}
bool fp_is_quadratic_residue_gpu(cudaStream_t s, uint32_t g, const Fp *a) {
  return fp_host(s, g, GM_FP_IS_QR, nullptr, a, nullptr, 0, "fp_is_quadratic_residue_gpu") != 0;
}
void fp_pow_u64_gpu(cudaStream_t s, uint32_t g, Fp *result, const Fp *base, uint64_t exp) {
  fp_host(s, g, GM_FP_POW_U64, result, base, nullptr, exp, "fp_pow_u64_gpu");
}

void fp2_add_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b) { fp2_host(GM_FP2_ADD, result, a, b, 0, "fp2_add_gpu"); }
void fp2_sub_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b) { fp2_host(GM_FP2_SUB, result, a, b, 0, "fp2_sub_gpu"); }
void fp2_mul_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b) { fp2_host(GM_FP2_MUL, result, a, b, 0, "fp2_mul_gpu"); }
void fp2_neg_gpu(Fp2 *result, const Fp2 *a) { fp2_host(GM_FP2_NEG, result, a, nullptr, 0, "fp2_neg_gpu"); }
void fp2_conjugate_gpu(Fp2 *result, const Fp2 *a) {
  fp2_host(GM_FP2_CONJUGATE, result, a, nullptr, 0, "fp2_conjugate_gpu");
}
void fp2_square_gpu(Fp2 *result, const Fp2 *a) { fp2_host(GM_FP2_SQUARE, result, a, nullptr, 0, "fp2_square_gpu"); }
void fp2_inv_gpu(Fp2 *result, const Fp2 *a) { fp2_host(GM_FP2_INV, result, a, nullptr, 0, "fp2_inv_gpu"); }
void fp2_div_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b) { fp2_host(GM_FP2_DIV, result, a, b, 0, "fp2_div_gpu"); }
void fp2_mul_by_i_gpu(Fp2 *result, const Fp2 *a) {
  fp2_host(GM_FP2_MUL_BY_I, result, a, nullptr, 0, "fp2_mul_by_i_gpu");
}
void fp2_frobenius_gpu(Fp2 *result, const Fp2 *a) {
  fp2_host(GM_FP2_FROBENIUS, result, a, nullptr, 0, "fp2_frobenius_gpu");
}
int fp2_cmp_gpu(const Fp2 *a, const Fp2 *b) { return fp2_host(GM_FP2_CMP, nullptr, a, b, 0, "fp2_cmp_gpu"); }
bool fp2_is_zero_gpu(const Fp2 *a) { return fp2_host(GM_FP2_IS_ZERO, nullptr, a, nullptr, 0, "fp2_is_zero_gpu") != 0; }
bool fp2_is_one_gpu(const Fp2 *a) { return fp2_host(GM_FP2_IS_ONE, nullptr, a, nullptr, 0, "fp2_is_one_gpu") != 0; }
void fp2_copy_gpu(Fp2 *result, const Fp2 *a) { fp2_host(GM_FP2_COPY, result, a, nullptr, 0, "fp2_copy_gpu"); }
void fp2_cmov_gpu(Fp2 *result, const Fp2 *src, uint64_t condition) {
  fp2_host(GM_FP2_CMOV, result, src, nullptr, condition, "fp2_cmov_gpu", true);
}
