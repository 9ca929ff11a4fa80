/*
 * gpu_msm_b200 -- the reference's C++ API for the MSM path.
 *
 * Declarations identical, name for name and signature for signature, to
 * pdroalves/gpu_msm include/curve.h:207-241 (MSM entry points, batched
 * Montgomery conversion, point at infinity), include/curve.h:108
 * (init_device_generators), include/fp_kernels.h:15-39 and
 * include/fp2_kernels.h:13-19 (field arrays).  The types are the
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

#endif /* GPU_MSM_B200_CXX_H */
