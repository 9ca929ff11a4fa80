/*
 * gpu_msm_b200 -- the point and field types shared by the C-ABI
 * (gpu_msm_b200.h) and the C++ API (gpu_msm_b200_cxx.h).
 */
#ifndef GPU_MSM_B200_TYPES_H
#define GPU_MSM_B200_TYPES_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Types: byte-compatible with include/fp.h:13, include/fp2.h:10 and
 * include/curve.h:13-43 of the reference (sizes 56/112/120/232/168/336 B). */
typedef struct Fp { uint64_t limb[7]; } Fp;
typedef struct Fp2 { Fp c0; Fp c1; } Fp2;
typedef struct G1Point { Fp x; Fp y; bool infinity; } G1Point;
typedef struct G2Point { Fp2 x; Fp2 y; bool infinity; } G2Point;
typedef struct G1ProjectivePoint { Fp X; Fp Y; Fp Z; } G1ProjectivePoint;
typedef struct G2ProjectivePoint { Fp2 X; Fp2 Y; Fp2 Z; } G2ProjectivePoint;

typedef struct CUstream_st *gm_stream_t; /* a cudaStream_t */

#ifdef __cplusplus
}
#endif
#endif /* GPU_MSM_B200_TYPES_H */
