// Element-wise Fp / Fp2 kernels: the Fp microbench (2^26 independent
// fp_mont_mul pairs) and the device-array entry points that replace
// fp_mul_array_device / fp2_mul_array_host (pdroalves/gpu_msm
// src/fp_kernels.cu:223, src/fp2_kernels.cu:165).
//
// One element per thread in a grid-stride loop over a grid sized to the SM
// count; elements are 56 B (Fp) / 112 B (Fp2) records read and written as
// u64 words, so a warp touches contiguous memory.  The kernels are IMAD-bound:
// 798 IMAD per Fp product against 168 B of traffic.
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/gpu_msm_b200.h"
#include "msm_engine.h"
#include "msm_kernels.cuh"

namespace {

enum Op { MONT_MUL = 0, NORMAL_MUL = 1, MONT_SQR = 2, ADD = 3 };

template <class F, int OP>
__global__ void __launch_bounds__(256) k_field_mul(uint64_t *__restrict__ c, const uint64_t *__restrict__ a,
                                                   const uint64_t *__restrict__ b, int64_t n) {
  constexpr int Hw = F::LIMBS / 2;
  using M = F;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    typename F::T x, y;
    gm::load_ref<F>(x, a + i * Hw);
    typename F::T z;
    if constexpr (OP == MONT_SQR) {
      z = F::sqr(x);
    } else if constexpr (OP == ADD) {
      gm::load_ref<F>(y, b + i * Hw);
      z = F::add(x, y);
    } else {
      gm::load_ref<F>(y, b + i * Hw);
      z = M::mul(x, y);
    }
    if (OP == NORMAL_MUL) {
      // (a*b*R^-1) * R^2 * R^-1 = a*b
      gm::fp_t r2;
#pragma unroll
      for (int k = 0; k < gm::NL; k++) r2.v[k] = gm::FpConst::R2(k);
      if constexpr (F::LIMBS == gm::NL) {
        z = M::mul(z, r2);
      } else {
        z.c0 = gm::Fp::mul(z.c0, r2);
        z.c1 = gm::Fp::mul(z.c1, r2);
      }
    }
    gm::store_ref<F>(c + i * Hw, z);
  }
}

int sm_count(int dev) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <class F, int OP>
int launch_field(gm_stream_t stream, uint32_t gpu_index, void *c, const void *a, const void *b, int64_t n) {
  if (n < 0 || (n > 0 && (c == nullptr || a == nullptr || b == nullptr))) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_field_mul<F, OP>, 256, 0);
  const int64_t max_blocks = (int64_t)sm_count((int)gpu_index) * (per_sm > 0 ? per_sm : 1);
  const int64_t need = (n + 255) / 256;
  const unsigned grid = (unsigned)(need < max_blocks ? need : max_blocks);
  k_field_mul<F, OP><<<grid, 256, 0, (cudaStream_t)stream>>>((uint64_t *)c, (const uint64_t *)a, (const uint64_t *)b, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_field_mul");
}

// IMAD-pipe throughput probe: 16 independent accumulator chains per thread.
// mode 0 issues 8 mad.lo.u32 + 8 mad.hi.u32 per iteration (the lo/hi mix of a
// Montgomery product), mode 1 issues 16 mad.lo.u32.  Each chain depends only
// on its own previous value.  Used to measure the integer multiply-add
// ceiling that the MSM roofline is quoted against.
__global__ void __launch_bounds__(256) k_imad_probe(uint32_t *__restrict__ sink, int iters, uint32_t seed, int mode) {
  uint32_t a[16];
#pragma unroll
  for (int k = 0; k < 16; k++) a[k] = seed * (threadIdx.x + 1) + 0x9e3779b9u * (k + 1);
  const uint32_t m = seed | 1u, c = seed ^ 0x85ebca6bu;
  if (mode == 0) {
    for (int it = 0; it < iters; it++) {
#pragma unroll
      for (int k = 0; k < 16; k += 2) {
        asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
        asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[k + 1]) : "r"(m), "r"(c));
      }
    }
  } else {
    for (int it = 0; it < iters; it++) {
#pragma unroll
      for (int k = 0; k < 16; k++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) x ^= a[k];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = x;
}

}  // namespace

extern "C" {

int gm_imad_probe(gm_stream_t stream, uint32_t gpu_index, int iters, int mode, uint32_t *d_sink,
                  int64_t sink_words, int64_t *imad_per_launch) {
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_imad_probe, 256, 0);
  const int64_t blocks = (int64_t)sm_count((int)gpu_index) * (per_sm > 0 ? per_sm : 1);
  if (blocks * 256 > sink_words || iters <= 0) return gm::GM_ERR_ARG;
  k_imad_probe<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_sink, iters, 0x2545f491u, mode);
  gm::count_launches(1);
  if (imad_per_launch) *imad_per_launch = blocks * 256 * (int64_t)iters * 16;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_imad_probe");
}

int gm_profile_enable(int on) {
  gm::profile_enable(on != 0);
  return gm::GM_OK;
}

int gm_profile_collect(char *names, int names_len, float *ms, int max) {
  return gm::profile_collect(names, names_len, ms, max);
}

int64_t gm_launch_count_reset(void) { return gm::launches_and_reset(); }

int gm_fp_mont_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n) {
  return launch_field<gm::Fp, MONT_MUL>(stream, gpu_index, d_c, d_a, d_b, n);
}
int gm_fp_mont_sqr_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, int64_t n) {
  return launch_field<gm::Fp, MONT_SQR>(stream, gpu_index, d_c, d_a, d_a, n);
}
int gm_fp_add_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n) {
  return launch_field<gm::Fp, ADD>(stream, gpu_index, d_c, d_a, d_b, n);
}
int gm_fp2_add_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n) {
  return launch_field<gm::Fp2, ADD>(stream, gpu_index, d_c, d_a, d_b, n);
}
int gm_fp_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp *d_c, const Fp *d_a, const Fp *d_b, int64_t n) {
  return launch_field<gm::Fp, NORMAL_MUL>(stream, gpu_index, d_c, d_a, d_b, n);
}
int gm_fp2_mont_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n) {
  return launch_field<gm::Fp2, MONT_MUL>(stream, gpu_index, d_c, d_a, d_b, n);
}
int gm_fp2_mul_array(gm_stream_t stream, uint32_t gpu_index, Fp2 *d_c, const Fp2 *d_a, const Fp2 *d_b, int64_t n) {
  return launch_field<gm::Fp2, NORMAL_MUL>(stream, gpu_index, d_c, d_a, d_b, n);
}

}  // extern "C"
