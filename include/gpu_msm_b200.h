/*
 * gpu_msm_b200 -- B200-native (sm_100a) BLS12-446 multi-scalar multiplication.
 *
 * C-ABI of the shared library libgpu_msm_b200.so.  Plain pointers and sizes,
 * no C++ or torch types in the signatures.
 *
 * Part 1 reproduces, name for name and signature for signature, the C-ABI that
 * pdroalves/gpu_msm exports to its Rust crate (rust-api/include/rust_wrapper.h,
 * bound by rust-api/src/ffi.rs:65-106), so an existing binding links against
 * this library unchanged.  Part 2 adds entry points the reference does not
 * have (full-width scalars, device-resident inputs, resident base tables,
 * batches).  Each declaration names the reference interface it replaces.
 *
 * Conventions (same as the reference unless stated):
 *   - Fp is 7 little-endian u64 limbs; points hold Montgomery-form
 *     coordinates (R = 2^448) unless a function says "standard form".
 *   - Affine points carry an `infinity` flag; projective points use Z = 0 for
 *     infinity.  Struct pad bytes are never read.
 *   - Scalars are little-endian u64 limbs, `scalar_limbs` per scalar, stored
 *     scalar-major (scalar i occupies limbs [i*scalar_limbs, (i+1)*scalar_limbs)).
 *   - MSM results are homogeneous projective points; (X, Y, Z) is a valid
 *     representation of the sum, not a specific one, so results are compared
 *     after conversion to affine.
 *   - Status codes of the int-returning functions: 0 ok, -1 bad size/argument,
 *     -2 stream creation failed, -3 allocation failed, -4 CUDA error,
 *     -5 device consistency check failed.
 */
#ifndef GPU_MSM_B200_H
#define GPU_MSM_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#include "gpu_msm_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================== */
/* Part 1: the reference C-ABI (rust-api/include/rust_wrapper.h)             */
/* ======================================================================== */

/* rust_wrapper.h:14 -- Z = 1 (Montgomery); infinity -> (0, 0, 0) */
void affine_to_projective_g1_wrapper(G1ProjectivePoint *proj, const G1Point *affine);
/* rust_wrapper.h:17 */
void affine_to_projective_g2_wrapper(G2ProjectivePoint *proj, const G2Point *affine);
/* rust_wrapper.h:20 -- x = X/Z, y = Y/Z (Montgomery); Z = 0 -> infinity */
void projective_to_affine_g1_wrapper(G1Point *affine, const G1ProjectivePoint *proj);
/* rust_wrapper.h:23 */
void projective_to_affine_g2_wrapper(G2Point *affine, const G2ProjectivePoint *proj);
/* rust_wrapper.h:26-35 */
void g1_point_at_infinity_wrapper(G1Point *point);
void g2_point_at_infinity_wrapper(G2Point *point);
void g1_projective_point_at_infinity_wrapper(G1ProjectivePoint *point);
void g2_projective_point_at_infinity_wrapper(G2ProjectivePoint *point);
/* rust_wrapper.h:38-41 */
bool g1_is_infinity_wrapper(const G1Point *point);
bool g2_is_infinity_wrapper(const G2Point *point);

/* rust_wrapper.h:45 (c_wrapper.cu:64-172): host buffers, u64 scalars.
 * Points arrive in STANDARD form and are converted to Montgomery on the
 * device (c_wrapper.cu:127).  Returns 0, or -1 when n <= 0. */
int g1_msm_wrapper(G1ProjectivePoint *result, const G1Point *points, const uint64_t *scalars, int n,
                   uint32_t gpu_index);
/* rust_wrapper.h:53 (c_wrapper.cu:175-258): host buffers, u64 scalars.
 * Points are taken as already in Montgomery form (no conversion,
 * c_wrapper.cu:223-224), as in the reference. */
int g2_msm_wrapper(G2ProjectivePoint *result, const G2Point *points, const uint64_t *scalars, int n,
                   uint32_t gpu_index);

/* rust_wrapper.h:63-65 (c_wrapper.cu:261-288) */
void g1_from_montgomery_wrapper(G1Point *result, const G1Point *point);
void g2_from_montgomery_wrapper(G2Point *result, const G2Point *point);
void fp_to_montgomery_wrapper(Fp *result, const Fp *value);

/* include/curve.h:108 (src/curve.cu:833); bound with C linkage by
 * rust-api/src/ffi.rs:67.  Kept for link compatibility: the generators are
 * compile-time constants here, so this only validates the device index. */
#ifndef GM_CXX_API_IMPL /* the C++-linkage twin is in gpu_msm_b200_cxx.h */
void init_device_generators(gm_stream_t stream, uint32_t gpu_index);
#endif

/* ======================================================================== */
/* Part 2: additive entry points                                             */
/* ======================================================================== */

/* Full-width host-buffer MSM.  Replaces point_msm<G1Point>/<G2Point>
 * (include/curve.h:238-241, src/curve.cu:2763-2826) for callers of the
 * C-ABI, which the reference restricts to u64 scalars.  points_montgomery != 0:
 * points are in Montgomery form; 0: standard form (converted on device).
 * 1 <= scalar_limbs <= 8.  n == 0 yields infinity. */
int g1_msm_limbs_wrapper(G1ProjectivePoint *result, const G1Point *points, const uint64_t *scalars,
                         int scalar_limbs, int n, uint32_t gpu_index, int points_montgomery);
int g2_msm_limbs_wrapper(G2ProjectivePoint *result, const G2Point *points, const uint64_t *scalars,
                         int scalar_limbs, int n, uint32_t gpu_index, int points_montgomery);

/* Host-buffer MSM, asynchronous on `stream`: the same computation as
 * g{1,2}_msm_limbs_wrapper, enqueued instead of waited for.  The scalar and
 * point copies from host memory, the MSM and the copy of the projective
 * result to *result (host memory) are all ordered on `stream`; the call
 * returns once they are enqueued.  The host buffers must stay valid, and
 * *result unread, until the stream has passed the call (synchronise the
 * stream or an event recorded after it).  With page-locked buffers the
 * copies overlap other work on the GPU, e.g. the previous MSM on another
 * stream; with pageable ones the copies block.  *err_flag (host, optional)
 * receives the device consistency flag (0 = ok) in the same order.  No
 * reference counterpart: the reference's host-buffer wrappers are
 * synchronous (rust-api/src/c_wrapper.cu:64-258). */
int gm_g1_msm_host_async(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *result, const G1Point *points,
                         const uint64_t *scalars, int scalar_limbs, int n, int points_montgomery, uint32_t *err_flag);
int gm_g2_msm_host_async(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *result, const G2Point *points,
                         const uint64_t *scalars, int scalar_limbs, int n, int points_montgomery, uint32_t *err_flag);

/* Device-pointer MSM, asynchronous on `stream`.  Replaces
 * point_msm_u64_async_g1/_g2 (include/curve.h:232-235; scalar_limbs = 1) and
 * point_msm_async<G1Point>/<G2Point> (include/curve.h:238) without the
 * caller-sized scratch buffer: workspace comes from a per-device stream-
 * ordered pool.  d_points: reference-layout affine points, Montgomery form. */
int gm_g1_msm_device(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, int n);
int gm_g2_msm_device(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, int n);

/* Same, with explicit window width c (2..20); 0 picks c from the cost
 * model.  Used by the autotuner and by parity tests that sweep c. */
int gm_g1_msm_device_c(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                       const uint64_t *d_scalars, int scalar_limbs, int n, int window_bits);
int gm_g2_msm_device_c(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                       const uint64_t *d_scalars, int scalar_limbs, int n, int window_bits);

/* MSM with an affine result (Montgomery form; infinity flag set for the
 * identity), the device form of point_msm_async<G1Point>/<G2Point>
 * (include/curve.h:238, src/curve.cu:2763), which returns an affine point.
 * Asynchronous: the projective sum is converted to affine by a host
 * function ordered on the stream.  n == 0 writes the point at infinity. */
int gm_g1_msm_device_affine(gm_stream_t stream, uint32_t gpu_index, G1Point *d_result, const G1Point *d_points,
                            const uint64_t *d_scalars, int scalar_limbs, int n);
int gm_g2_msm_device_affine(gm_stream_t stream, uint32_t gpu_index, G2Point *d_result, const G2Point *d_points,
                            const uint64_t *d_scalars, int scalar_limbs, int n);

/* G1 MSM that allocates nothing.  No counterpart in the reference.  For
 * callers that cannot allocate device memory per call: frameworks that hand
 * almost all of HBM to their own caching allocator, and latency-critical code
 * that must not take the implicit synchronisation of cudaMalloc/cudaFree.
 * Same arguments and result as gm_g1_msm_device, but the workspace is a fixed
 * 8 MiB array in the library's device image, reserved on every GPU that loads
 * the library until the process exits.  Limit: n <= 4096 points and
 * 1 <= scalar_limbs <= 8; larger requests return -1 without launching.  All
 * calls share the array: calls that overlap on the GPU race, so order them on
 * one stream.  The first call on a device looks up the array's address on
 * that device; make it before any stream capture there.  d_err (device
 * pointer, may be NULL) receives, on the stream, the pipeline's consistency
 * flag: 0, or non-zero if the result must not be trusted (the regular
 * blocking wrappers return -5 in that case). */
int gm_g1_msm_device_noalloc(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result,
                             const G1Point *d_points, const uint64_t *d_scalars, int scalar_limbs, int n,
                             uint32_t *d_err);

/* Resident base tables and batched MSMs.  No reference counterpart: every
 * reference MSM copies and converts its bases again (c_wrapper.cu:64-172).
 *
 * gm_bases_create: packs n reference-layout points (device pointer; Montgomery
 *   form when points_montgomery != 0, else standard form, converted) into an
 *   owned device table on gpu_index; blocks until done.  n < 2^31.
 * gm_msm_resident: one MSM over table entries [base_offset, base_offset + n),
 *   asynchronous on `stream`; result is one projective point of the table's
 *   group.  window_bits 0 = cost model.
 * gm_batch_plan_create: fixes a batch of `count` MSMs: MSM i uses table
 *   entries [base_offsets[i], base_offsets[i] + sizes[i]) (base_offsets may be
 *   NULL: all 0) and window width window_bits[i] (NULL or 0: cost model).
 *   MSMs of equal width form a class that runs as one flattened pipeline on
 *   its own stream.  All workspace is allocated here.
 * gm_batch_plan_run: enqueues the batch on `stream` (forks the classes and
 *   joins them back): d_scalars holds the MSMs' scalar rows concatenated in
 *   MSM order, scalar_limbs u64 each; d_results receives `count` projective
 *   points in MSM order.  Only kernels, memsets and event waits are enqueued.
 * gm_batch_plan_classes: window width and MSM count of each class.
 * gm_batch_run: the same batch without a plan: workspace and descriptors come
 *   from the per-device stream-ordered pool for this one run and the classes
 *   run in order on `stream` (for batches whose shape changes every time, as
 *   in serving).
 * gm_batch_run_ws: gm_batch_run in the caller's device workspace
 *   (d_workspace, 256-byte aligned, workspace_bytes at least
 *   gm_batch_workspace_bytes of the batch; GM_ERR_ARG otherwise), so that a
 *   server that keeps one workspace per in-flight batch takes no pool
 *   allocation per batch.  The workspace is in use until the stream has run
 *   the batch.  No counterpart in the reference.
 * gm_batch_workspace_bytes: device bytes gm_batch_run takes for that batch
 *   (for admission control), or -1 on a bad argument. */
typedef struct gm_bases gm_bases;
typedef struct gm_batch_plan gm_batch_plan;
int gm_bases_create(uint32_t gpu_index, int group, const void *d_points, int64_t n, int points_montgomery,
                    gm_bases **out);
int gm_bases_destroy(gm_bases *bases);
/* Fixed-base window table of a resident set: for window width c =
 * window_bits, stores 2^(c w) * P_i for every point and every window w that
 * scalars of scalar_limbs limbs need (64 * scalar_limbs / c + 1), in affine
 * Montgomery form.  Afterwards MSMs over the set (gm_msm_resident, batches,
 * plans) whose window width is c use one bucket set for all windows and no
 * window doublings; MSMs without an explicit width pick the cheapest table.
 * Memory: n * W records (128 B G1, 256 B G2).  Blocks until built; calling
 * it again for a width that is already there does nothing.  No counterpart in
 * the reference. */
int gm_bases_precompute(gm_bases *b, int window_bits, int scalar_limbs);
int64_t gm_bases_count(const gm_bases *bases);
int gm_msm_resident(gm_stream_t stream, const gm_bases *bases, int64_t base_offset, int n, const uint64_t *d_scalars,
                    int scalar_limbs, void *d_result, int window_bits);
int gm_batch_plan_create(const gm_bases *bases, int scalar_limbs, int count, const int64_t *sizes,
                         const int64_t *base_offsets, const int32_t *window_bits, gm_batch_plan **out);
int gm_batch_plan_run(gm_batch_plan *plan, gm_stream_t stream, const uint64_t *d_scalars, void *d_results);
/* gm_batch_plan_create with per-MSM tuning (no reference counterpart):
 * tuning[2 i] = accumulation slices of MSM i's window class in resident waves
 * of threads (1, 2 or 4; 0 = 1), tuning[2 i + 1] = pass-A sort tile in points
 * per thread (2, 4 or 8, i.e. 512, 1024 or 2048 points; 0 = 4).  A class
 * takes the values of its largest MSM.  NULL tuning = gm_batch_plan_create.
 * The autotuner (gpu_msm_b200/autotune.py) picks them per size class. */
int gm_batch_plan_create_tuned(const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                               const int64_t *base_offsets, const int32_t *window_bits, const int32_t *tuning,
                               gm_batch_plan **out);

/* Accumulation mode of a plan (no reference counterpart): 1 (default) = the
 * accumulation of every window class in one persistent launch over a device
 * work queue of (class, 32 slices) items, between the classes' sorts and
 * their fix-ups; 0 = one pipeline per window class, each on its own stream
 * with full-GPU kernels.  Results are identical; the mode only changes
 * scheduling. */
int gm_batch_plan_set_queue(gm_batch_plan *p, int on);
int gm_batch_plan_destroy(gm_batch_plan *plan);
int64_t gm_batch_plan_bytes(const gm_batch_plan *plan);
int gm_batch_plan_classes(const gm_batch_plan *plan, int32_t *window_bits, int32_t *counts, int max);
int gm_batch_run(gm_stream_t stream, const gm_bases *bases, int scalar_limbs, int count, const int64_t *sizes,
                 const int64_t *base_offsets, const int32_t *window_bits, const uint64_t *d_scalars, void *d_results);
int gm_batch_run_ws(gm_stream_t stream, const gm_bases *bases, int scalar_limbs, int count, const int64_t *sizes,
                    const int64_t *base_offsets, const int32_t *window_bits, const uint64_t *d_scalars,
                    void *d_results, void *d_workspace, int64_t workspace_bytes);
int64_t gm_batch_workspace_bytes(const gm_bases *bases, int scalar_limbs, int count, const int64_t *sizes,
                                 const int32_t *window_bits);

/* Window width the cost model picks for an MSM of n points (group 1 or 2). */
int gm_msm_default_window(int group, int64_t n, int scalar_limbs);

/* Fp microbench kernels (device pointers, asynchronous).
 * gm_fp_mont_mul_array: c[i] = a[i]*b[i]*R^-1 (Montgomery form), the
 *   batched form of fp_mont_mul (src/fp.cu:370).
 * gm_fp_mul_array: c[i] = a[i]*b[i] mod p on standard-form values, the
 *   C-ABI form of fp_mul_array_device (include/fp_kernels.h:39).
 * gm_fp_mont_sqr_array: c[i] = a[i]^2*R^-1, the dedicated Montgomery squaring
 *   used inside the point formulas (same result as fp_mont_mul(a, a),
 *   src/fp.cu:370; the reference has no separate squaring).
 * gm_fp2_mont_mul_array: batched fp2_mont_mul (src/fp2.cu:88).
 * gm_fp2_mul_array: batched normal-form fp2_mul on device pointers, the
 *   device-resident form of fp2_mul_array_host (include/fp2_kernels.h:19). */
int gm_fp_mont_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n);
int gm_fp_mont_sqr_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, int64_t n);
/* c[i] = a[i] + b[i] mod p (either form); the device form of
 * fp_add_array_device (include/fp_kernels.h:33) and fp2_add_array_host
 * (include/fp2_kernels.h:13). */
int gm_fp_add_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n);
int gm_fp2_add_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n);
int gm_fp_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n);
int gm_fp2_mont_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n);
int gm_fp2_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n);

/* Batched standard <-> Montgomery conversion of reference-layout affine
 * points in place (device pointers).  Replaces point_to_montgomery_batch
 * (include/curve.h:207, src/curve.cu:2506); from_montgomery has no batched
 * counterpart in the reference (src/curve.cu:2356 is never launched). */
int gm_g1_to_montgomery_batch(gm_stream_t stream, uint32_t gpu_index, G1Point *d_points, int n);
int gm_g2_to_montgomery_batch(gm_stream_t stream, uint32_t gpu_index, G2Point *d_points, int n);

/* Fixed-base batch: out[i] = k_i * G (Montgomery affine, canonical), for the
 * generator G of src/curve.cu:786-814.  No reference counterpart beyond the
 * single-point point_scalar_mul (src/curve.cu:230); used to build synthetic
 * base tables P_i = k_i * G on the device. */
int gm_g1_generator_mul_batch(gm_stream_t stream, uint32_t gpu_index, G1Point *d_out, const uint64_t *d_scalars,
                              int scalar_limbs, int n);
int gm_g2_generator_mul_batch(gm_stream_t stream, uint32_t gpu_index, G2Point *d_out, const uint64_t *d_scalars,
                              int scalar_limbs, int n);

/* d_out = sum of n projective points (device pointers, one thread).  Adds
 * the partial MSM results of shards computed on several devices or in
 * several batches; the reference has no sharded MSM. */
int gm_g1_sum_projective(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_out,
                         const G1ProjectivePoint *d_in, int n);
int gm_g2_sum_projective(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_out,
                         const G2ProjectivePoint *d_in, int n);

/* Self-test of the host arithmetic of the window combination (Montgomery
 * squaring against the general product, Jacobian-doubling Horner against the
 * XYZZ one); 0 when every check passes.  No reference counterpart. */
int gm_host_selftest(void);

/* Single-element operations on device pointers, asynchronous on `stream`:
 * the C-ABI behind the reference's stream APIs fp_*_async
 * (include/fp.h:158-204), fp2_*_async (include/fp2.h:99-133) and
 * point_*_async<G1Point|G2Point> (include/curve.h:156-211), and behind its
 * host-pointer helpers (include/fp_kernels.h:26-38, include/fp2_kernels.h:21-37).
 *
 * gm_fp_elem / gm_fp2_elem: c = op(a, b).  MUL, INV, DIV, SQUARE, SQRT, IS_QR
 *   and POW_U64 work on standard-form values (the reference's fp_mul,
 *   fp_inv, ... convert to and from Montgomery form inside); MONT_MUL is the
 *   Montgomery product; inverses and quotients of 0 are 0.  CMOV: c = a when
 *   (arg & 1), else c is left as it is.  POW_U64: c = a^arg.  CMP writes
 *   -1 / 0 / 1 (limb-wise comparison, c0 before c1 for Fp2) to *d_flag;
 *   IS_ZERO, IS_ONE and IS_QR write 0 / 1 there; SQRT writes c and 0 / 1
 *   (a^((p+1)/4) for a quadratic residue, else c = 0 and 0).
 * gm_g{1,2}_point_elem: affine points in Montgomery form.  ADD, DOUBLE, NEG
 *   follow the reference's affine formulas and branch order
 *   (src/curve.cu:72-227); SCALAR_MUL takes scalar_limbs little-endian u64
 *   limbs at d_scalar, SCALAR_MUL_U64 the value scalar_u64; TO_MONT /
 *   FROM_MONT convert both coordinates (infinity -> zeros + flag);
 *   AT_INFINITY writes the identity.
 * Inputs are canonical field elements (below p).  Returns -1 for an unknown
 * op or a missing pointer the op needs. */
enum {
  GM_FP_ADD = 0,
  GM_FP_SUB = 1,
  GM_FP_MUL = 2,
  GM_FP_NEG = 3,
  GM_FP_INV = 4,
  GM_FP_DIV = 5,
  GM_FP_COPY = 6,
  GM_FP_ZERO = 7,
  GM_FP_ONE = 8,
  GM_FP_TO_MONT = 9,
  GM_FP_FROM_MONT = 10,
  GM_FP_MONT_MUL = 11,
  GM_FP_CMP = 12,
  GM_FP_IS_ZERO = 13,
  GM_FP_IS_ONE = 14,
  GM_FP_CMOV = 15,
  GM_FP_SQRT = 16,
  GM_FP_IS_QR = 17,
  GM_FP_POW_U64 = 18,
  GM_FP_OP_COUNT = 19
};
enum {
  GM_FP2_ADD = 0,
  GM_FP2_SUB = 1,
  GM_FP2_MUL = 2,
  GM_FP2_SQUARE = 3,
  GM_FP2_NEG = 4,
  GM_FP2_CONJUGATE = 5,
  GM_FP2_INV = 6,
  GM_FP2_DIV = 7,
  GM_FP2_COPY = 8,
  GM_FP2_MUL_BY_I = 9,
  GM_FP2_FROBENIUS = 10,
  GM_FP2_CMP = 11,
  GM_FP2_IS_ZERO = 12,
  GM_FP2_IS_ONE = 13,
  GM_FP2_CMOV = 14,
  GM_FP2_MONT_MUL = 15,
  GM_FP2_OP_COUNT = 16
};
enum {
  GM_PT_ADD = 0,
  GM_PT_DOUBLE = 1,
  GM_PT_NEG = 2,
  GM_PT_SCALAR_MUL = 3,
  GM_PT_SCALAR_MUL_U64 = 4,
  GM_PT_TO_MONT = 5,
  GM_PT_FROM_MONT = 6,
  GM_PT_AT_INFINITY = 7,
  GM_PT_OP_COUNT = 8
};
int gm_fp_elem(gm_stream_t stream, uint32_t gpu_index, int op, Fp *d_c, const Fp *d_a, const Fp *d_b, uint64_t arg,
               int32_t *d_flag);
int gm_fp2_elem(gm_stream_t stream, uint32_t gpu_index, int op, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b,
                uint64_t arg, int32_t *d_flag);
int gm_g1_point_elem(gm_stream_t stream, uint32_t gpu_index, int op, G1Point *d_r, const G1Point *d_p,
                     const G1Point *d_q, const uint64_t *d_scalar, int scalar_limbs, uint64_t scalar_u64);
int gm_g2_point_elem(gm_stream_t stream, uint32_t gpu_index, int op, G2Point *d_r, const G2Point *d_p,
                     const G2Point *d_q, const uint64_t *d_scalar, int scalar_limbs, uint64_t scalar_u64);

/* d_ok[i] = 1 when affine point i (Montgomery form, device pointers) lies on
 * the curve -- y^2 = x^3 + 1 (G1), y^2 = x^3 + (1 + i) (G2), the equations
 * the reference's generators satisfy -- or carries the infinity flag; else 0.
 * The reference's is_on_curve_g1/g2 (include/curve.h:53-59) are host/device
 * inline functions with b = 4 / 4i, which reject its own generators; this
 * batched check uses the corrected constants.  Validates bases before they
 * become a resident table. */
int gm_g1_on_curve_batch(gm_stream_t stream, uint32_t gpu_index, const G1Point *d_points, int64_t n, uint8_t *d_ok);
int gm_g2_on_curve_batch(gm_stream_t stream, uint32_t gpu_index, const G2Point *d_points, int64_t n, uint8_t *d_ok);

/* Host-side sum of n G1 projective points (Montgomery form): combines the
 * partial results of a sharded MSM on a CPU; no reference counterpart. */
int gm_g1_sum_projective_host(G1ProjectivePoint *out, const G1ProjectivePoint *in, int n);

/* Measurement hooks (no reference counterpart).
 * gm_profile_enable: while on, every MSM records CUDA events on its stream at
 *   its phase boundaries (pack, sort, accumulate, fixup, reduce, combine).
 * gm_profile_collect: waits for those events and returns up to `max`
 *   per-phase milliseconds in launch order, with their names comma-separated
 *   in `names`; clears the record.
 * gm_launch_count_reset: number of kernels this library launched from the
 *   calling thread since the previous call.
 * gm_imad_probe: launches a kernel of independent multiply-add chains over
 *   the whole GPU (mode 0: half mad.lo, half mad.hi, the mix of an integer
 *   Montgomery product; mode 1: mad.lo only); *imad_per_launch receives the instruction
 *   count so that the caller can time it and derive the ceiling. */
int gm_profile_enable(int on);
int gm_profile_collect(char *names, int names_len, float *ms, int max);
int64_t gm_launch_count_reset(void);
int gm_imad_probe(gm_stream_t stream, uint32_t gpu_index, int iters, int mode, uint32_t *d_sink,
                  int64_t sink_words, int64_t *imad_per_launch);

/* Last CUDA error string seen by this library on the calling thread. */
const char *gm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* GPU_MSM_B200_H */
