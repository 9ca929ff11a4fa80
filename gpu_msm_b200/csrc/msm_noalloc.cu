// G1 MSM that allocates nothing: its workspace is a fixed array in device
// memory that belongs to the library image, not to any allocator.
//
// Who needs it: callers that cannot allocate device memory per call.  A
// framework that hands (almost) all of HBM to its own caching allocator
// leaves nothing for cudaMalloc/cudaMallocAsync; real-time or latency-
// critical callers cannot afford the implicit device synchronisation and
// unbounded latency of cudaMalloc/cudaFree; some runtimes forbid allocation
// outright once they are set up.  This entry point calls no cudaMalloc,
// cudaFree, pool or pinned-host allocation, and no allocating library routine.
//
// Limits and contract:
//   * at most NOALLOC_MAX_POINTS points and NOALLOC_MAX_LIMBS scalar limbs per
//     call; larger requests are rejected with GM_ERR_ARG before any launch;
//   * the scratch array (NOALLOC_SCRATCH_BYTES) is reserved on every GPU
//     that loads the library, for the life of the process;
//   * every call uses the same array and leaves the last call's contents in
//     it; the parts that must start at zero are cleared on the stream by
//     each call.  Calls whose work overlaps on the GPU (different streams
//     without ordering, or different host threads) race on the array and
//     give wrong results: order them on one stream, or serialise them;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make
//     that first call before any stream capture on that device;
//   * the pipeline is the regular one (msm_run: the same sort, accumulation,
//     fix-up, reduction and device window combination), planned with a fixed
//     window width and a fixed number of accumulation slices so that its
//     workspace never depends on the GPU; the fix-up's consistency flag goes
//     to the caller's d_err, like the regular asynchronous entry points'.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gpu_msm_b200.h"
#include "msm_host.cuh"

namespace gm {
// instantiated once, in msm_g1.cu
extern template int msm_plan<Fp>(MsmLayout<Fp> &, int, int64_t, int, int, bool, int64_t);
extern template int msm_run<Fp>(cudaStream_t, const MsmLayout<Fp> &, char *, const uint4 *, const uint64_t *, int,
                                const uint64_t *, uint64_t *, bool, uint32_t *, cudaEvent_t, TailHandoff *);
}  // namespace gm

namespace {

constexpr int64_t NOALLOC_MAX_POINTS = 4096;
constexpr int NOALLOC_MAX_LIMBS = 8;
constexpr int NOALLOC_WINDOW_BITS = 8;
// accumulation slices: bounds the slice partials whatever the GPU's SM count
constexpr int64_t NOALLOC_SLICE_THREADS = 4096;
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_addr_mu;
void *g_addr[64] = {nullptr};

// Device address of the scratch array on `dev` (the current device).  The
// array's name in host code is only a stand-in and must never reach a kernel.
int scratch_address(int dev, void **out) {
  if (dev < 0 || dev >= 64) {
    gm::set_last_error("device index out of range for the no-alloc scratch table");
    return gm::GM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (g_addr[dev] == nullptr) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return gm::record_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return gm::GM_OK;
}

}  // namespace

extern "C" int gm_g1_msm_device_noalloc(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result,
                                        const G1Point *d_points, const uint64_t *d_scalars, int scalar_limbs, int n,
                                        uint32_t *d_err) {
  using gm::Fp;
  if (d_result == nullptr || n < 0 || (n > 0 && (d_points == nullptr || d_scalars == nullptr))) {
    gm::set_last_error("gm_g1_msm_device_noalloc: null pointer or negative size");
    return gm::GM_ERR_ARG;
  }
  if (n > NOALLOC_MAX_POINTS || scalar_limbs < 1 || scalar_limbs > NOALLOC_MAX_LIMBS) {
    gm::set_last_error("gm_g1_msm_device_noalloc: at most 4096 points and 1..8 scalar limbs per call");
    return gm::GM_ERR_ARG;
  }
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  constexpr int H = Fp::LIMBS / 2;
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(d_result, 0, 3 * H * sizeof(uint64_t), s);
    if (e == cudaSuccess && d_err) e = cudaMemsetAsync(d_err, 0, sizeof(uint32_t), s);
    return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "cudaMemsetAsync(result)");
  }
  void *base = nullptr;
  rc = scratch_address((int)gpu_index, &base);
  if (rc) return rc;
  gm::MsmLayout<Fp> lay;
  rc = gm::msm_plan<Fp>(lay, (int)gpu_index, n, scalar_limbs, NOALLOC_WINDOW_BITS, /*pack=*/true,
                        NOALLOC_SLICE_THREADS);
  if (rc) return rc;
  if (lay.bytes > NOALLOC_SCRATCH_BYTES) {
    gm::set_last_error("gm_g1_msm_device_noalloc: request exceeds the fixed scratch size");
    return gm::GM_ERR_ARG;
  }
  // the same pipeline as the regular entry points, in the fixed array, with
  // the window combination on the device (the host tail needs pinned memory)
  return gm::msm_run<Fp>(s, lay, static_cast<char *>(base), nullptr, (const uint64_t *)d_points, 0, d_scalars,
                         (uint64_t *)d_result, /*host_tail=*/false, d_err, nullptr);
}
