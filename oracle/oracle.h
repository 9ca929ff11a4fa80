/*
 * CPU oracle for the BLS12-446 MSM path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's host arithmetic
 * (pdroalves/gpu_msm: src/fp.cu, src/fp2.cu, src/curve.cu).  It exists so
 * that tests, the smoke check and the CPU-baseline leg of bench.py can check
 * the CUDA library against the reference algorithm.  Nothing in the product
 * path (gpu_msm_b200/) may link or call it.
 *
 * Parity pin: the restatement is checked against the reference's own
 * known-answer tests (tests/test_fp.cu, tests/test_fp2.cu, tests/test_msm.cu)
 * through tests/golden/, and against the reference host code itself compiled
 * by oracle/Makefile into oracle/_ref/ (when the reference sources are
 * present on the build machine).
 *
 * Struct layouts are byte-compatible with the reference types
 * (include/fp.h:13, include/fp2.h:10, include/curve.h:13-43).
 */
#ifndef GPU_MSM_ORACLE_H
#define GPU_MSM_ORACLE_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_LIMBS 7

typedef struct { uint64_t limb[ORC_LIMBS]; } orc_fp;          /* 56 B  */
typedef struct { orc_fp c0, c1; } orc_fp2;                     /* 112 B */
typedef struct { orc_fp x, y; bool infinity; } orc_g1;        /* 120 B */
typedef struct { orc_fp2 x, y; bool infinity; } orc_g2;       /* 232 B */
typedef struct { orc_fp X, Y, Z; } orc_g1p;                   /* 168 B */
typedef struct { orc_fp2 X, Y, Z; } orc_g2p;                  /* 336 B */

/* ---- Fp (src/fp.cu) ---------------------------------------------------- */
void orc_fp_add(orc_fp *c, const orc_fp *a, const orc_fp *b);
void orc_fp_sub(orc_fp *c, const orc_fp *a, const orc_fp *b);
void orc_fp_neg(orc_fp *c, const orc_fp *a);
void orc_fp_mont_mul(orc_fp *c, const orc_fp *a, const orc_fp *b);
void orc_fp_to_mont(orc_fp *c, const orc_fp *a);
void orc_fp_from_mont(orc_fp *c, const orc_fp *a);
void orc_fp_mul(orc_fp *c, const orc_fp *a, const orc_fp *b);
void orc_fp_inv(orc_fp *c, const orc_fp *a);
void orc_fp_mont_inv(orc_fp *c, const orc_fp *a);
void orc_fp_pow(orc_fp *c, const orc_fp *a, const uint64_t *e, int e_limbs);

/* batch helpers over arrays (for ctypes) */
void orc_fp_mont_mul_batch(orc_fp *c, const orc_fp *a, const orc_fp *b, int64_t n);
void orc_fp_mul_batch(orc_fp *c, const orc_fp *a, const orc_fp *b, int64_t n);
void orc_fp_to_mont_batch(orc_fp *c, const orc_fp *a, int64_t n);
void orc_fp_from_mont_batch(orc_fp *c, const orc_fp *a, int64_t n);

/* ---- Fp2 (src/fp2.cu) -------------------------------------------------- */
void orc_fp2_add(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b);
void orc_fp2_sub(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b);
void orc_fp2_mont_mul(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b);
void orc_fp2_mul(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b);
void orc_fp2_mont_inv(orc_fp2 *c, const orc_fp2 *a);
void orc_fp2_mont_mul_batch(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b, int64_t n);
void orc_fp2_mul_batch(orc_fp2 *c, const orc_fp2 *a, const orc_fp2 *b, int64_t n);

/* ---- curve (src/curve.cu), all coordinates in Montgomery form ----------- */
void orc_g1_generator(orc_g1 *g_standard);
void orc_g2_generator(orc_g2 *g_standard);
void orc_g1_to_mont(orc_g1 *r, const orc_g1 *p);
void orc_g2_to_mont(orc_g2 *r, const orc_g2 *p);
void orc_g1_from_mont(orc_g1 *r, const orc_g1 *p);
void orc_g2_from_mont(orc_g2 *r, const orc_g2 *p);

void orc_g1_add(orc_g1 *r, const orc_g1 *a, const orc_g1 *b);
void orc_g1_double(orc_g1 *r, const orc_g1 *a);
void orc_g1_scalar_mul(orc_g1 *r, const orc_g1 *p, const uint64_t *k, int limbs);
void orc_g2_add(orc_g2 *r, const orc_g2 *a, const orc_g2 *b);
void orc_g2_double(orc_g2 *r, const orc_g2 *a);
void orc_g2_scalar_mul(orc_g2 *r, const orc_g2 *p, const uint64_t *k, int limbs);

void orc_g1p_add(orc_g1p *r, const orc_g1p *a, const orc_g1p *b);
void orc_g1p_double(orc_g1p *r, const orc_g1p *a);
void orc_g2p_add(orc_g2p *r, const orc_g2p *a, const orc_g2p *b);
void orc_g2p_double(orc_g2p *r, const orc_g2p *a);
void orc_g1_affine_to_proj(orc_g1p *r, const orc_g1 *a);
void orc_g2_affine_to_proj(orc_g2p *r, const orc_g2 *a);
void orc_g1_proj_to_affine(orc_g1 *r, const orc_g1p *a);
void orc_g2_proj_to_affine(orc_g2 *r, const orc_g2p *a);

/* projective double-and-add (same canonical result as the affine
 * point_scalar_mul of src/curve.cu:230, one inversion at the end) */
void orc_g1_scalar_mul_fast(orc_g1 *r, const orc_g1 *p, const uint64_t *k, int limbs);
void orc_g2_scalar_mul_fast(orc_g2 *r, const orc_g2 *p, const uint64_t *k, int limbs);

/* ---- MSM oracles: output canonical affine (Montgomery form) ------------ */
/* reference-structured Pippenger: 4-bit unsigned windows, projective
 * buckets, combine_buckets_cpu_projective per window (src/curve.cu:2060). */
void orc_g1_msm_pippenger(orc_g1 *r, const orc_g1 *pts, const uint64_t *scalars,
                          int limbs, int64_t n, int threads);
void orc_g2_msm_pippenger(orc_g2 *r, const orc_g2 *pts, const uint64_t *scalars,
                          int limbs, int64_t n, int threads);
/* naive: sum_i k_i * P_i by double-and-add per term */
void orc_g1_msm_naive(orc_g1 *r, const orc_g1 *pts, const uint64_t *scalars,
                      int limbs, int64_t n, int threads);
void orc_g2_msm_naive(orc_g2 *r, const orc_g2 *pts, const uint64_t *scalars,
                      int limbs, int64_t n, int threads);

/* on-curve checks with the curve constants the generators satisfy:
 * b = 1 (G1), b' = 1 + i (G2).  Inputs in Montgomery form. */
bool orc_g1_on_curve(const orc_g1 *p);
bool orc_g2_on_curve(const orc_g2 *p);

#ifdef __cplusplus
}
#endif
#endif
