// MSM launch sequence (templated on the field), instantiated once per group
// in msm_g1.cu / msm_g2.cu so the two large kernel sets compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

#include "msm_engine.h"
#include "msm_kernels.cuh"

namespace gm {

static inline int windows_for(int c, int limbs) { return (64 * limbs) / c + 1; }
#define GM_CHECK(call)                                     \
  do {                                                     \
    cudaError_t _e = (call);                               \
    if (_e != cudaSuccess) return record_error(_e, #call); \
  } while (0)

#define GM_CHECK_LAUNCH(where)                             \
  do {                                                     \
    cudaError_t _e = cudaGetLastError();                   \
    if (_e != cudaSuccess) return record_error(_e, where); \
  } while (0)

// ---------------------------------------------------------------------------
// workspace layout
// ---------------------------------------------------------------------------
static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Carve {
  size_t off = 0;
  template <class T>
  size_t take(size_t count) {
    const size_t o = align_up(off, 256);
    off = o + count * sizeof(T);
    return o;
  }
};

template <class F>
struct MsmLayout {
  DigitParams dp;
  int64_t K = 0, nthreads = 0, n = 0;
  int L1 = 8;     // buckets per reduction segment
  int FAN = 4;    // fan-in of the segment-share tree
  int nseg = 0;   // reduction segments per window
  size_t o_counts, o_offsets, o_bsum, o_entries, o_buckets, o_head, o_tail, o_hk, o_tk, o_red[3], o_err, o_packed;
  size_t bytes = 0;
  int64_t nb = 0;
  int64_t red_elems = 0;
  bool need_pack = false;

  void plan(int64_t n_, int limbs, int c, int sms, int acc_blocks_per_sm, bool pack) {
    n = n_;
    need_pack = pack;
    dp.c = c;
    dp.W = windows_for(c, limbs);
    dp.B = 1 << (c - 1);
    dp.limbs = limbs;
    K = (int64_t)dp.W * dp.B;
    nb = (K + SCAN_TILE - 1) / SCAN_TILE;
    nthreads = (int64_t)sms * std::max(1, acc_blocks_per_sm) * ACC_THREADS;
    // never more slices than entries
    const int64_t max_entries = n * dp.W;
    if (nthreads > max_entries) nthreads = std::max<int64_t>(1, (max_entries + 127) / 128 * 128);
    L1 = std::min(L1, dp.B);
    nseg = (dp.B + L1 - 1) / L1;
    red_elems = (int64_t)dp.W * nseg;
    Carve cv;
    o_counts = cv.take<uint32_t>(K);
    o_offsets = cv.take<uint32_t>(K + 1);
    o_bsum = cv.take<uint32_t>(nb);
    o_entries = cv.take<uint32_t>((size_t)std::max<int64_t>(1, max_entries));
    o_buckets = cv.take<xyzz_t<F>>(K);
    o_head = cv.take<xyzz_t<F>>(nthreads);
    o_tail = cv.take<xyzz_t<F>>(nthreads);
    o_hk = cv.take<int32_t>(nthreads);
    o_tk = cv.take<int32_t>(nthreads);
    o_red[0] = cv.take<xyzz_t<F>>(red_elems);
    o_red[1] = cv.take<xyzz_t<F>>((red_elems + FAN - 1) / FAN + dp.W);
    o_red[2] = cv.take<xyzz_t<F>>((red_elems + FAN - 1) / FAN + dp.W);
    o_err = cv.take<uint32_t>(4);
    o_packed = pack ? cv.take<uint4>((size_t)n * Rec<F>::U4) : 0;
    bytes = cv.off;
  }
};

// Blocks of k_accumulate resident per SM; the dynamic shared-memory opt-in is
// a per-device function attribute, so it is set (and cached) per device.
template <class F>
static int acc_blocks_per_sm(int dev) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int b = 0;
    cudaFuncSetAttribute(k_accumulate<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, acc_smem_bytes<F>());
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_accumulate<F>, ACC_THREADS, acc_smem_bytes<F>()) !=
        cudaSuccess)
      b = 1;
    cached[dev] = std::max(1, b);
  }
  return cached[dev];
}

static inline unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

// Runs the whole pipeline.  bases: packed records (or null to pack from
// ref_points), scalars: device u64 limbs, out: reference projective layout.
template <class F>
int msm_launch(cudaStream_t s, int dev, const uint4 *bases, const uint64_t *ref_points, int to_mont,
               const uint64_t *scalars, int limbs, int64_t n, uint64_t *out_proj, int c_override,
               uint32_t *err_out) {
  constexpr int H = F::LIMBS / 2;  // u64 words per coordinate
  if (n == 0) {
    GM_CHECK(cudaMemsetAsync(out_proj, 0, 3 * H * sizeof(uint64_t), s));
    return GM_OK;
  }
  if (limbs < 1 || limbs > MAX_SCALAR_LIMBS || n < 0 || n > (int64_t)INT32_MAX) {
    set_last_error("invalid scalar_limbs or n");
    return GM_ERR_ARG;
  }
  int sms = 0;
  int rc = device_sm_count(dev, &sms);
  if (rc) return rc;
  const int c = c_override > 0 ? c_override : default_window(sizeof(typename F::T) == sizeof(fp_t) ? 1 : 2, n, limbs);
  if (c < 2 || c > 20) {
    set_last_error("window width out of range");
    return GM_ERR_ARG;
  }
  MsmLayout<F> lay;
  lay.plan(n, limbs, c, sms, acc_blocks_per_sm<F>(dev), bases == nullptr);
  if ((uint64_t)n * lay.dp.W >= (1ull << 32)) {
    set_last_error("too many (point, window) entries for 32-bit offsets");
    return GM_ERR_ARG;
  }
  char *ws = nullptr;
  rc = pool_alloc(dev, s, lay.bytes, (void **)&ws);
  if (rc) return rc;

  auto *counts = (uint32_t *)(ws + lay.o_counts);
  auto *offsets = (uint32_t *)(ws + lay.o_offsets);
  auto *bsum = (uint32_t *)(ws + lay.o_bsum);
  auto *entries = (uint32_t *)(ws + lay.o_entries);
  auto *buckets = (xyzz_t<F> *)(ws + lay.o_buckets);
  auto *head = (xyzz_t<F> *)(ws + lay.o_head);
  auto *tail = (xyzz_t<F> *)(ws + lay.o_tail);
  auto *hk = (int32_t *)(ws + lay.o_hk);
  auto *tk = (int32_t *)(ws + lay.o_tk);
  auto *err = (uint32_t *)(ws + lay.o_err);
  xyzz_t<F> *red[3];
  for (int k = 0; k < 3; k++) red[k] = (xyzz_t<F> *)(ws + lay.o_red[k]);

  profile_mark(s, "start");
  int launches = 0;
  if (bases == nullptr) {
    uint4 *packed = (uint4 *)(ws + lay.o_packed);
    k_pack_ref<F><<<grid_for(n, 256), 256, 0, s>>>(packed, ref_points, n, 2 * H + 1, to_mont);
    GM_CHECK_LAUNCH("k_pack_ref");
    bases = packed;
    launches++;
    profile_mark(s, "pack");
  }
  GM_CHECK(cudaMemsetAsync(counts, 0, lay.K * sizeof(uint32_t), s));
  GM_CHECK(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  k_count<<<grid_for(n, 256), 256, 0, s>>>(scalars, bases, Rec<F>::U4, F::LIMBS, n, lay.dp, counts);
  GM_CHECK_LAUNCH("k_count");
  k_scan_blocksum<<<(unsigned)lay.nb, SCAN_THREADS, 0, s>>>(counts, lay.K, bsum);
  k_scan_top<<<1, SCAN_THREADS, 0, s>>>(bsum, (int)lay.nb);
  k_scan_final<<<(unsigned)lay.nb, SCAN_THREADS, 0, s>>>(counts, lay.K, bsum, offsets);
  GM_CHECK_LAUNCH("k_scan");
  k_scatter<<<grid_for(n, 256), 256, 0, s>>>(scalars, bases, Rec<F>::U4, F::LIMBS, n, lay.dp, offsets, counts,
                                             entries);
  GM_CHECK_LAUNCH("k_scatter");
  launches += 5;
  profile_mark(s, "sort");
  k_accumulate<F><<<grid_for(lay.nthreads, ACC_THREADS), ACC_THREADS, acc_smem_bytes<F>(), s>>>(bases, entries, offsets, lay.K, lay.nthreads, buckets,
                                                               head, tail, hk, tk);
  GM_CHECK_LAUNCH("k_accumulate");
  launches++;
  profile_mark(s, "accumulate");
  k_fixup<F><<<grid_for(lay.nthreads, 128), 128, 0, s>>>(offsets, lay.K, lay.nthreads, buckets, head, tail, hk, tk, err);
  GM_CHECK_LAUNCH("k_fixup");
  launches++;
  profile_mark(s, "fixup");

  // bucket reduction: per-segment shares, then a fan-in tree per window
  const int W = lay.dp.W;
  {
    const int64_t th = (int64_t)W * lay.nseg;
    k_reduce_segments<F><<<grid_for(th, 128), 128, 0, s>>>(buckets, offsets, W, lay.dp.B, lay.L1, red[0]);
    GM_CHECK_LAUNCH("k_reduce_segments");
    launches++;
  }
  int N = lay.nseg;
  xyzz_t<F> *src = red[0];
  int pong = 1;
  while (N > 1) {
    const int nout = (N + lay.FAN - 1) / lay.FAN;
    xyzz_t<F> *dst = red[pong];
    k_tree_sum<F><<<grid_for((int64_t)W * nout, 128), 128, 0, s>>>(src, W, N, lay.FAN, dst);
    GM_CHECK_LAUNCH("k_tree_sum");
    launches++;
    src = dst;
    pong = pong == 1 ? 2 : 1;
    N = nout;
  }
  profile_mark(s, "reduce");
  // window combination: the serial Horner tail runs on the host (lower
  // latency per product) unless the stream is being captured into a graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GM_CHECK(cudaStreamIsCapturing(s, &cap));
  if (cap == cudaStreamCaptureStatusNone && host_tail_enabled()) {
    rc = enqueue_host_tail(s, F::LIMBS == NL ? 1 : 2, src, W, c, out_proj);
    if (rc) return rc;
  } else {
    k_combine<F><<<1, 32, 0, s>>>(src, 1, W, c, out_proj);
    GM_CHECK_LAUNCH("k_combine");
    launches++;
  }
  profile_mark(s, "combine");
  count_launches(launches);
  if (err_out) GM_CHECK(cudaMemcpyAsync(err_out, err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  GM_CHECK(cudaFreeAsync(ws, s));
  return GM_OK;
}

}  // namespace gm
