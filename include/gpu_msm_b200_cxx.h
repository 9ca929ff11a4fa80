/*
 * gpu_msm_b200 -- the reference's C++ API for the MSM path.
 *
 * Declarations identical, name for name and signature for signature, to
 * pdroalves/gpu_msm include/curve.h:156-241 (MSM entry points, single-point
 * stream operations, batched Montgomery conversion, point at infinity),
 * include/curve.h:108 (init_device_generators), include/fp.h:158-204 and
 * include/fp2.h:99-133 (single-element stream operations),
 * include/fp_kernels.h and include/fp2_kernels.h (field arrays and the
 * host-pointer single-element helpers).  The types are the
 * byte-compatible structs of gpu_msm_b200_types.h, so the mangled symbols
 * match the reference's and object files built against its headers link
 * against libgpu_msm_b200.so unchanged.
 *
 * Behaviour follows the reference:
 *   - device pointers, asynchronous on `stream` unless the name has no
 *     `_async` (those synchronise the stream before returning);
 *   - bases in Montgomery form, scalars as little-endian u64 limbs
 *     (scalar_limbs per scalar, scalar-major), n == 0 gives the identity;
 *   - invalid arguments or CUDA errors print a message and abort(), as the
 *     reference's PANIC_IF_FALSE / check_cuda_error do (include/device.h);
 *   - `d_scratch` must be non-null like in the reference but is not used:
 *     the workspace comes from the library's stream-ordered pool.
 */
#ifndef GPU_MSM_B200_CXX_H
#define GPU_MSM_B200_CXX_H

#ifndef __cplusplus
#error "gpu_msm_b200_cxx.h is a C++ header; C callers use gpu_msm_b200.h"
#endif

#include <cuda_runtime.h>

#include <cstdint>

#include "gpu_msm_b200_types.h"

/* include/curve.h:108 */
void init_device_generators(cudaStream_t stream, uint32_t gpu_index);

/* include/curve.h:232-235: u64 scalars, projective result */
void point_msm_u64_async_g1(cudaStream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result,
                            const G1Point *d_points, const uint64_t *d_scalars, G1ProjectivePoint *d_scratch, int n);
void point_msm_u64_g1(cudaStream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                      const uint64_t *d_scalars, G1ProjectivePoint *d_scratch, int n);
void point_msm_u64_async_g2(cudaStream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result,
                            const G2Point *d_points, const uint64_t *d_scalars, G2ProjectivePoint *d_scratch, int n);
void point_msm_u64_g2(cudaStream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                      const uint64_t *d_scalars, G2ProjectivePoint *d_scratch, int n);

/* include/curve.h:238-241: multi-limb scalars, affine result
 * (instantiated for G1Point and G2Point) */
template <typename PointType>
void point_msm_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, PointType *d_scratch, int n);
template <typename PointType>
void point_msm(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_points,
               const uint64_t *d_scalars, int scalar_limbs, PointType *d_scratch, int n);

/* include/curve.h:203-208: standard -> Montgomery form in place */
template <typename PointType>
void point_to_montgomery_batch_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_points, int n);
template <typename PointType>
void point_to_montgomery_batch(cudaStream_t stream, uint32_t gpu_index, PointType *d_points, int n);

/* include/curve.h:190-192 */
template <typename PointType>
void point_at_infinity_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result);
template <typename PointType>
void point_at_infinity(cudaStream_t stream, uint32_t gpu_index, PointType *d_result);

extern template void point_msm_async<G1Point>(cudaStream_t, uint32_t, G1Point *, const G1Point *, const uint64_t *,
                                              int, G1Point *, int);
extern template void point_msm<G1Point>(cudaStream_t, uint32_t, G1Point *, const G1Point *, const uint64_t *, int,
                                        G1Point *, int);
extern template void point_msm_async<G2Point>(cudaStream_t, uint32_t, G2Point *, const G2Point *, const uint64_t *,
                                              int, G2Point *, int);
extern template void point_msm<G2Point>(cudaStream_t, uint32_t, G2Point *, const G2Point *, const uint64_t *, int,
                                        G2Point *, int);
extern template void point_to_montgomery_batch_async<G1Point>(cudaStream_t, uint32_t, G1Point *, int);
extern template void point_to_montgomery_batch<G1Point>(cudaStream_t, uint32_t, G1Point *, int);
extern template void point_to_montgomery_batch_async<G2Point>(cudaStream_t, uint32_t, G2Point *, int);
extern template void point_to_montgomery_batch<G2Point>(cudaStream_t, uint32_t, G2Point *, int);
extern template void point_at_infinity_async<G1Point>(cudaStream_t, uint32_t, G1Point *);
extern template void point_at_infinity<G1Point>(cudaStream_t, uint32_t, G1Point *);
extern template void point_at_infinity_async<G2Point>(cudaStream_t, uint32_t, G2Point *);
extern template void point_at_infinity<G2Point>(cudaStream_t, uint32_t, G2Point *);

/* include/fp_kernels.h:15-39: element-wise products (normal form) and sums;
 * _host variants take host pointers and synchronise, _device variants take
 * device pointers and are asynchronous */
void fp_add_array_host(cudaStream_t stream, uint32_t gpu_index, Fp *c, const Fp *a, const Fp *b, int n);
void fp_mul_array_host(cudaStream_t stream, uint32_t gpu_index, Fp *c, const Fp *a, const Fp *b, int n);
void fp_add_array_device(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int n);
void fp_mul_array_device(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int n);

/* include/fp2_kernels.h:13-19 */
void fp2_add_array_host(cudaStream_t stream, uint32_t gpu_index, Fp2 *c, const Fp2 *a, const Fp2 *b, int n);
void fp2_mul_array_host(cudaStream_t stream, uint32_t gpu_index, Fp2 *c, const Fp2 *a, const Fp2 *b, int n);

/* include/fp.h:158-204: single-element Fp operations on device pointers.
 * mul, inv, div work on standard-form values; mont_mul on Montgomery form;
 * inv(0) = 0, x / 0 = 0; one() is the standard-form 1. */
void fp_add_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_add(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_sub_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_sub(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_mul_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_mul(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_neg_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_neg(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_inv_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_inv(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_div_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_div(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_copy_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_dst, const Fp *d_src);
void fp_copy(cudaStream_t stream, uint32_t gpu_index, Fp *d_dst, const Fp *d_src);
void fp_zero_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_a);
void fp_zero(cudaStream_t stream, uint32_t gpu_index, Fp *d_a);
void fp_one_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_a);
void fp_one(cudaStream_t stream, uint32_t gpu_index, Fp *d_a);
void fp_to_montgomery_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_to_montgomery(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_from_montgomery_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_from_montgomery(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a);
void fp_mont_mul_async(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);
void fp_mont_mul(cudaStream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b);

/* include/fp2.h:99-133: single-element Fp2 operations on device pointers
 * (mul, square, inv, div on standard-form values) */
void fp2_add_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_add(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_sub_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_sub(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_mul_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_mul(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_square_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_square(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_neg_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_neg(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_conjugate_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_conjugate(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_inv_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_inv(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a);
void fp2_div_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_div(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b);
void fp2_copy_async(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_dst, const Fp2 *d_src);
void fp2_copy(cudaStream_t stream, uint32_t gpu_index, Fp2 *d_dst, const Fp2 *d_src);

/* include/curve.h:156-205: single-point operations on device pointers,
 * affine Montgomery-form points (instantiated for G1Point and G2Point) */
template <typename PointType>
void point_add_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p1,
                     const PointType *d_p2);
template <typename PointType>
void point_add(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p1,
               const PointType *d_p2);
template <typename PointType>
void point_double_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p);
template <typename PointType>
void point_double(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p);
template <typename PointType>
void point_neg_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p);
template <typename PointType>
void point_neg(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_p);
template <typename PointType>
void point_scalar_mul_u64_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result,
                                const PointType *d_point, uint64_t scalar);
template <typename PointType>
void point_scalar_mul_u64(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                          uint64_t scalar);
template <typename PointType>
void point_scalar_mul_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                            const uint64_t *d_scalar, int scalar_limbs);
template <typename PointType>
void point_scalar_mul(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point,
                      const uint64_t *d_scalar, int scalar_limbs);
template <typename PointType>
void point_to_montgomery_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result,
                               const PointType *d_point);
template <typename PointType>
void point_to_montgomery(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point);
template <typename PointType>
void point_from_montgomery_async(cudaStream_t stream, uint32_t gpu_index, PointType *d_result,
                                 const PointType *d_point);
template <typename PointType>
void point_from_montgomery(cudaStream_t stream, uint32_t gpu_index, PointType *d_result, const PointType *d_point);

#define GM_CXX_POINT_EXTERN(P)                                                                                \
  extern template void point_add_async<P>(cudaStream_t, uint32_t, P *, const P *, const P *);                 \
  extern template void point_add<P>(cudaStream_t, uint32_t, P *, const P *, const P *);                       \
  extern template void point_double_async<P>(cudaStream_t, uint32_t, P *, const P *);                         \
  extern template void point_double<P>(cudaStream_t, uint32_t, P *, const P *);                               \
  extern template void point_neg_async<P>(cudaStream_t, uint32_t, P *, const P *);                            \
  extern template void point_neg<P>(cudaStream_t, uint32_t, P *, const P *);                                  \
  extern template void point_scalar_mul_u64_async<P>(cudaStream_t, uint32_t, P *, const P *, uint64_t);       \
  extern template void point_scalar_mul_u64<P>(cudaStream_t, uint32_t, P *, const P *, uint64_t);             \
  extern template void point_scalar_mul_async<P>(cudaStream_t, uint32_t, P *, const P *, const uint64_t *, int); \
  extern template void point_scalar_mul<P>(cudaStream_t, uint32_t, P *, const P *, const uint64_t *, int);    \
  extern template void point_to_montgomery_async<P>(cudaStream_t, uint32_t, P *, const P *);                  \
  extern template void point_to_montgomery<P>(cudaStream_t, uint32_t, P *, const P *);                        \
  extern template void point_from_montgomery_async<P>(cudaStream_t, uint32_t, P *, const P *);                \
  extern template void point_from_montgomery<P>(cudaStream_t, uint32_t, P *, const P *);
GM_CXX_POINT_EXTERN(G1Point)
GM_CXX_POINT_EXTERN(G2Point)
#undef GM_CXX_POINT_EXTERN

/* include/fp_kernels.h:26-38: one Fp operation on HOST pointers (copied to
 * the device, run, copied back, stream synchronised) */
void fp_add_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a, const Fp *b);
void fp_sub_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a, const Fp *b);
void fp_mul_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a, const Fp *b);
void fp_neg_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
void fp_inv_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
void fp_div_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a, const Fp *b);
int fp_cmp_gpu(cudaStream_t stream, uint32_t gpu_index, const Fp *a, const Fp *b);
bool fp_is_zero_gpu(cudaStream_t stream, uint32_t gpu_index, const Fp *a);
bool fp_is_one_gpu(cudaStream_t stream, uint32_t gpu_index, const Fp *a);
void fp_to_montgomery_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
void fp_from_montgomery_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
void fp_mont_mul_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a, const Fp *b);
void fp_copy_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
void fp_cmov_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *src, uint64_t condition);
bool fp_sqrt_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *a);
bool fp_is_quadratic_residue_gpu(cudaStream_t stream, uint32_t gpu_index, const Fp *a);
void fp_pow_u64_gpu(cudaStream_t stream, uint32_t gpu_index, Fp *result, const Fp *base, uint64_t exp);

/* include/fp2_kernels.h:21-37: one Fp2 operation on HOST pointers, on the
 * current device and the default stream */
void fp2_add_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b);
void fp2_sub_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b);
void fp2_mul_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b);
void fp2_neg_gpu(Fp2 *result, const Fp2 *a);
void fp2_conjugate_gpu(Fp2 *result, const Fp2 *a);
void fp2_square_gpu(Fp2 *result, const Fp2 *a);
void fp2_inv_gpu(Fp2 *result, const Fp2 *a);
void fp2_div_gpu(Fp2 *result, const Fp2 *a, const Fp2 *b);
void fp2_mul_by_i_gpu(Fp2 *result, const Fp2 *a);
void fp2_frobenius_gpu(Fp2 *result, const Fp2 *a);
int fp2_cmp_gpu(const Fp2 *a, const Fp2 *b);
bool fp2_is_zero_gpu(const Fp2 *a);
bool fp2_is_one_gpu(const Fp2 *a);
void fp2_copy_gpu(Fp2 *result, const Fp2 *a);
void fp2_cmov_gpu(Fp2 *result, const Fp2 *src, uint64_t condition);

#endif /* GPU_MSM_B200_CXX_H */
