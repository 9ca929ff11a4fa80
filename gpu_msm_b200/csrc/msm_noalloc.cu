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
//     that first call before any stream capture on that device.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gpu_msm_b200.h"
#include "msm_host.cuh"

namespace {

constexpr int64_t NOALLOC_MAX_POINTS = 4096;
constexpr int NOALLOC_MAX_LIMBS = 8;
constexpr int NOALLOC_WINDOW_BITS = 8;
constexpr int NOALLOC_SLICE_THREADS = 4096;  // accumulation slices (bounds the partials)
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

unsigned grid_of(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

extern "C" int gm_g1_msm_device_noalloc(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result,
                                        const G1Point *d_points, const uint64_t *d_scalars, int scalar_limbs,
                                        int n) {
  using gm::Fp;
  using gm::xyzz_t;
  using gm::record_error;
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
    return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "cudaMemsetAsync(result)");
  }
  void *base = nullptr;
  rc = scratch_address((int)gpu_index, &base);
  if (rc) return rc;

  // workspace layout inside the fixed array; planned for NOALLOC_SLICE_THREADS
  // accumulation slices so the slice partials stay small
  gm::MsmLayout<Fp> lay;
  lay.plan(n, scalar_limbs, NOALLOC_WINDOW_BITS, NOALLOC_SLICE_THREADS / gm::ACC_THREADS, 1, /*pack=*/true);
  if (lay.bytes > NOALLOC_SCRATCH_BYTES) {
    gm::set_last_error("gm_g1_msm_device_noalloc: request exceeds the fixed scratch size");
    return gm::GM_ERR_ARG;
  }
  // sets the accumulation kernel's dynamic shared-memory attribute (no allocation)
  (void)gm::acc_blocks_per_sm<Fp>((int)gpu_index, false);

  char *ws = static_cast<char *>(base);
  auto *counts = (uint32_t *)(ws + lay.o_counts);
  auto *offsets = (uint32_t *)(ws + lay.o_offsets);
  auto *bsum = (uint32_t *)(ws + lay.o_bsum);
  auto *entries = (uint32_t *)(ws + lay.o_entries);
  auto *buckets = (xyzz_t<Fp> *)(ws + lay.o_buckets);
  auto *head = (xyzz_t<Fp> *)(ws + lay.o_head);
  auto *tail = (xyzz_t<Fp> *)(ws + lay.o_tail);
  auto *hk = (int32_t *)(ws + lay.o_hk);
  auto *tk = (int32_t *)(ws + lay.o_tk);
  auto *err = (uint32_t *)(ws + lay.o_err);
  auto *packed = (uint4 *)(ws + lay.o_packed);
  xyzz_t<Fp> *red[3];
  for (int k = 0; k < 3; k++) red[k] = (xyzz_t<Fp> *)(ws + lay.o_red[k]);

  // what must start at zero: the bucket counters and the consistency flag
  GM_CHECK(cudaMemsetAsync(counts, 0, lay.K * sizeof(uint32_t), s));
  GM_CHECK(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  gm::k_pack_ref<Fp><<<grid_of(n, 256), 256, 0, s>>>(packed, (const uint64_t *)d_points, n, 2 * H + 1, 0);
  GM_CHECK_LAUNCH("k_pack_ref");
  gm::k_count<<<grid_of(n, 256), 256, 0, s>>>(d_scalars, n, lay.dp, counts);
  GM_CHECK_LAUNCH("k_count");
  gm::k_scan_blocksum<<<(unsigned)lay.nb, gm::SCAN_THREADS, 0, s>>>(counts, lay.K, bsum);
  gm::k_scan_top<<<1, gm::SCAN_THREADS, 0, s>>>(bsum, (int)lay.nb);
  gm::k_scan_final<<<(unsigned)lay.nb, gm::SCAN_THREADS, 0, s>>>(counts, lay.K, bsum, offsets);
  GM_CHECK_LAUNCH("k_scan");
  gm::k_scatter<<<grid_of(n, 256), 256, 0, s>>>(d_scalars, n, lay.dp, offsets, counts, entries);
  GM_CHECK_LAUNCH("k_scatter");
  gm::k_accumulate<Fp><<<grid_of(lay.nthreads, gm::ACC_THREADS), gm::ACC_THREADS, gm::acc_smem_bytes<Fp>(), s>>>(
      packed, entries, offsets, lay.K, lay.nthreads, buckets, head, tail, hk, tk);
  GM_CHECK_LAUNCH("k_accumulate");
  gm::k_fixup<Fp><<<grid_of(lay.nthreads, 128), 128, 0, s>>>(offsets, lay.K, lay.nthreads, buckets, head, tail, hk,
                                                              tk, err);
  GM_CHECK_LAUNCH("k_fixup");
  const int W = lay.dp.W;
  gm::k_reduce_segments<Fp><<<grid_of((int64_t)W * lay.nseg, 128), 128, 0, s>>>(buckets, offsets, W, lay.dp.B,
                                                                                lay.L1, red[0]);
  GM_CHECK_LAUNCH("k_reduce_segments");
  int launches = 9;
  int N = lay.nseg, pong = 1;
  xyzz_t<Fp> *src = red[0];
  while (N > 1) {
    const int nout = (N + lay.FAN - 1) / lay.FAN;
    gm::k_tree_sum<Fp><<<grid_of((int64_t)W * nout, 128), 128, 0, s>>>(src, W, N, lay.FAN, red[pong]);
    GM_CHECK_LAUNCH("k_tree_sum");
    launches++;
    src = red[pong];
    pong = pong == 1 ? 2 : 1;
    N = nout;
  }
  // window combination on the device (the host tail would need pinned memory)
  gm::k_combine<Fp><<<1, 32, 0, s>>>(src, 1, W, NOALLOC_WINDOW_BITS, (uint64_t *)d_result);
  GM_CHECK_LAUNCH("k_combine");
  gm::count_launches(launches + 1);
  return gm::GM_OK;
}
