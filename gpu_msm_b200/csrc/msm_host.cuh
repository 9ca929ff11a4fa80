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
#include "msm_reduce.cuh"
#include "msm_sort.cuh"

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
  size_t o_offsets, o_entries, o_buckets, o_head, o_tail, o_hk, o_tk, o_err, o_packed, o_longq;
  size_t bytes = 0;
  int64_t long_cap = 0;
  bool need_pack = false;
  SortLayout sl;
  RedLayout rl;

  // slice_threads: accumulation slices (one per thread of a single wave);
  // level0_wave / coop_wave: threads of k_red_level0 / k_red_level1 resident
  // at once
  void plan(int64_t n_, int limbs, int c, int64_t slice_threads, bool pack, int64_t level0_wave,
            int64_t coop_wave) {
    n = n_;
    need_pack = pack;
    dp.c = c;
    dp.W = windows_for(c, limbs);
    dp.B = 1 << (c - 1);
    dp.limbs = limbs;
    K = (int64_t)dp.W * dp.B;
    nthreads = std::max<int64_t>(ACC_THREADS, slice_threads);
    // never more slices than entries
    const int64_t max_entries = n * dp.W;
    if (nthreads > max_entries) nthreads = std::max<int64_t>(1, (max_entries + 127) / 128 * 128);
    Carve cv;
    o_offsets = cv.take<uint32_t>(K + 1);
    o_entries = cv.take<uint32_t>((size_t)std::max<int64_t>(1, max_entries));
    sl.plan(dp, 1, n, (n + SA_TP - 1) / SA_TP, /*tabled=*/false, cv);
    o_buckets = cv.take<xyzz_t<F>>(K);
    o_head = cv.take<xyzz_t<F>>(nthreads);
    o_tail = cv.take<xyzz_t<F>>(nthreads);
    o_hk = cv.take<int32_t>(nthreads);
    o_tk = cv.take<int32_t>(nthreads);
    rl.plan<F>(dp.W, dp.B, level0_wave, cv, coop_wave);
    long_cap = nthreads / FIX_SHORT + 1;
    o_longq = cv.take<int32_t>((size_t)(1 + long_cap));
    o_err = cv.take<uint32_t>(4);
    o_packed = pack ? cv.take<uint4>((size_t)n * Rec<F>::U4) : 0;
    bytes = cv.off;
  }
};

// k_accumulate runs at most ACC_BLOCKS_MAX blocks per SM.  Its slices carry
// equal work, so a block that shares its SM with more blocks than the others
// finishes late and holds up the whole launch: with 3 blocks per SM the G1
// 2^20 accumulation took 13.8 ms against 13.3 ms, and batches, whose classes'
// launches overlap, 196 ms against 143 ms.  The grid holds ACC_BLOCKS_MAX
// blocks per SM, and where the registers would let more blocks share an SM
// the launch asks for enough dynamic shared memory to keep them out.
constexpr int ACC_BLOCKS_MAX = 2;

struct AccOccupancy {
  int blocks = 0;     // resident blocks per SM the grid is sized for
  size_t smem = 0;    // dynamic shared memory of a launch
};

// which: 0 = k_accumulate<F>, 1 = k_accumulate_queue<F> (same limits)
template <class F>
static AccOccupancy acc_occupancy(int dev, int which = 0) {
  static std::mutex mu;
  static AccOccupancy cached[2][64];
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) dev = 0;
  AccOccupancy &o = cached[which][dev];
  const void *fn = which == 0 ? (const void *)k_accumulate<F> : (const void *)k_accumulate_queue<F>;
  if (o.blocks == 0) {
    size_t smem = acc_smem_bytes<F>();
    int per_sm_smem = 0, b = 0;
    cudaDeviceGetAttribute(&per_sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, ACC_THREADS, smem) != cudaSuccess) b = 1;
    if (b > ACC_BLOCKS_MAX && per_sm_smem > 0) {
      // (ACC_BLOCKS_MAX + 1) blocks must not fit in the SM's shared memory
      const size_t pad = (size_t)per_sm_smem / (ACC_BLOCKS_MAX + 1) + 1024;
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pad) == cudaSuccess) smem = pad;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, ACC_THREADS, smem) != cudaSuccess) b = 1;
    }
    o.smem = smem;
    o.blocks = std::max(1, std::min(b, ACC_BLOCKS_MAX));
  }
  return o;
}

template <class F>
static int acc_blocks_per_sm(int dev) {
  return acc_occupancy<F>(dev).blocks;
}

template <class F>
static void acc_launch(unsigned grid, cudaStream_t s, const uint4 *bases, const uint32_t *entries,
                       const uint32_t *offsets, int64_t K, int64_t nthreads, xyzz_t<F> *buckets, xyzz_t<F> *head,
                       xyzz_t<F> *tail, int32_t *hk, int32_t *tk) {
  int dev = 0;
  cudaGetDevice(&dev);
  k_accumulate<F><<<grid, ACC_THREADS, acc_occupancy<F>(dev).smem, s>>>(bases, entries, offsets, K, nthreads,
                                                                          buckets, head, tail, hk, tk);
}

static inline unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

// Resident blocks per SM of the level-0 reduction kernel (cached per device).
template <class F>
static int level0_blocks_per_sm(int dev) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_red_level0<F>, 128, 0) != cudaSuccess) b = 1;
    cached[dev] = std::max(1, b);
  }
  return cached[dev];
}

// Threads of the cooperative level-1 reduction kernel resident at once on
// the device (cached per device).
template <class F>
static int64_t coop_wave_threads(int dev, int sms) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_red_level1<F>, 128, 0) != cudaSuccess) b = 1;
    cached[dev] = std::max(1, b);
  }
  return (int64_t)sms * cached[dev] * 128;
}

// Split fix-up: short runs serially, long runs by a block-level tree.
// long_q[0] must be zero on entry.
template <class F>
int fixup_launch(cudaStream_t s, const uint32_t *offsets, int64_t K, int64_t nthreads, xyzz_t<F> *buckets,
                 const xyzz_t<F> *head, const xyzz_t<F> *tail, const int32_t *hk, const int32_t *tk, uint32_t *err,
                 int32_t *long_q, int64_t long_cap, int *launches) {
  k_fixup_split<F><<<grid_for(nthreads, 128), 128, 0, s>>>(offsets, K, nthreads, buckets, head, tail, hk, tk, err,
                                                            long_q, long_cap);
  GM_CHECK_LAUNCH("k_fixup_split");
  k_fixup_long<F><<<FIX_LONG_BLOCKS, 128, 0, s>>>(offsets, K, nthreads, buckets, head, tail, hk, err, long_q,
                                                   long_cap);
  GM_CHECK_LAUNCH("k_fixup_long");
  *launches += 2;
  return GM_OK;
}

// Leveled bucket reduction over rl.G groups of rl.B buckets; *sums receives
// the G window sums (contiguous).
template <class F>
int reduce_launch(cudaStream_t s, const RedLayout &rl, const xyzz_t<F> *buckets, const uint32_t *offsets, char *ws,
                  const xyzz_t<F> **sums, int *launches) {
  auto *X = (xyzz_t<F> *)(ws + rl.o_X);
  auto *A0 = (xyzz_t<F> *)(ws + rl.o_A0);
  const int64_t wave = (int64_t)rl.sms * level0_blocks_per_sm<F>(rl.dev);
  const int64_t blocks0 = std::min<int64_t>(wave, (rl.G * rl.nseg0 + 127) / 128);
  k_red_level0<F><<<(unsigned)std::max<int64_t>(1, blocks0), 128, 0, s>>>(buckets, offsets, rl.G, rl.B, rl.L0,
                                                                           rl.nseg0, X, rl.M, A0);
  GM_CHECK_LAUNCH("k_red_level0");
  (*launches)++;
  if (rl.nseg1 > 0) {
    k_red_level1<F><<<grid_for((int64_t)Coop<F>::LANES * rl.G * rl.nseg1, 128), 128, 0, s>>>(A0, rl.G, rl.nseg0, rl.L1, rl.nseg1,
                                                                        rl.L0, X, rl.M);
    GM_CHECK_LAUNCH("k_red_level1");
    (*launches)++;
  }
  const xyzz_t<F> *src = X;
  int N = rl.M, k = 0;
  while (N > 1) {
    const int nout = (N + RedLayout::FAN - 1) / RedLayout::FAN;
    auto *dst = (xyzz_t<F> *)(ws + rl.o_t[k]);
    k_tree_quad<F><<<grid_for((int64_t)Coop<F>::LANES * rl.G * nout, 128), 128, 0, s>>>(src, rl.G, N, RedLayout::FAN, dst);
    GM_CHECK_LAUNCH("k_tree_quad");
    (*launches)++;
    src = dst;
    k ^= 1;
    N = nout;
  }
  *sums = src;
  return GM_OK;
}

// Plans the workspace of one MSM on device dev.  slice_threads 0: one
// accumulation slice per thread of a full wave (ACC_BLOCKS_MAX blocks per SM).
template <class F>
int msm_plan(MsmLayout<F> &lay, int dev, int64_t n, int limbs, int c, bool pack, int64_t slice_threads) {
  if (limbs < 1 || limbs > MAX_SCALAR_LIMBS || n < 1 || n > (int64_t)INT32_MAX) {
    set_last_error("invalid scalar_limbs or n");
    return GM_ERR_ARG;
  }
  if (c < 2 || c > 20) {
    set_last_error("window width out of range");
    return GM_ERR_ARG;
  }
  int sms = 0;
  int rc = device_sm_count(dev, &sms);
  if (rc) return rc;
  if (slice_threads <= 0) slice_threads = (int64_t)sms * acc_blocks_per_sm<F>(dev) * ACC_THREADS;
  lay.plan(n, limbs, c, slice_threads, pack, (int64_t)sms * level0_blocks_per_sm<F>(dev) * 128,
           coop_wave_threads<F>(dev, sms));
  lay.rl.sms = sms;
  lay.rl.dev = dev;
  if ((uint64_t)n * lay.dp.W >= (1ull << 32)) {
    set_last_error("too many (point, window) entries for 32-bit offsets");
    return GM_ERR_ARG;
  }
  return GM_OK;
}

// Enqueues the whole pipeline of one planned MSM on s, in the workspace ws
// (lay.bytes, 256-byte aligned); allocates nothing itself.  bases: packed
// records, or null to pack from ref_points (reference layout; to_mont converts
// standard-form points).  out_proj receives the projective result in the
// reference layout.  host_tail: the window combination runs on the host (a
// pinned staging slot and a stream-ordered host function); otherwise, and
// always while s is being captured, on the device.  err_out (optional,
// device) receives the consistency flag of the fix-up (0 = ok).  bases_ready
// (optional): an event the stream waits for after the sort, before the bases
// are first read.  handoff (optional): the window sums are copied to the
// caller's pinned buffer instead, and out_proj is not written.
template <class F>
int msm_run(cudaStream_t s, const MsmLayout<F> &lay, char *ws, const uint4 *bases, const uint64_t *ref_points,
            int to_mont, const uint64_t *scalars, uint64_t *out_proj, bool host_tail, uint32_t *err_out,
            cudaEvent_t bases_ready, TailHandoff *handoff = nullptr) {
  constexpr int H = F::LIMBS / 2;  // u64 words per coordinate
  const int64_t n = lay.n;
  auto *offsets = (uint32_t *)(ws + lay.o_offsets);
  auto *entries = (uint32_t *)(ws + lay.o_entries);
  auto *buckets = (xyzz_t<F> *)(ws + lay.o_buckets);
  auto *head = (xyzz_t<F> *)(ws + lay.o_head);
  auto *tail = (xyzz_t<F> *)(ws + lay.o_tail);
  auto *hk = (int32_t *)(ws + lay.o_hk);
  auto *tk = (int32_t *)(ws + lay.o_tk);
  auto *err = (uint32_t *)(ws + lay.o_err);
  auto *long_q = (int32_t *)(ws + lay.o_longq);
  profile_mark(s, "start");
  int launches = 0;
  // the sort needs only the scalars; the bases are packed after it, so a
  // caller that is still copying them in can overlap that copy with the sort
  GM_CHECK(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  GM_CHECK(cudaMemsetAsync(long_q, 0, sizeof(int32_t), s));
  {
    SortDesc sd;
    sd.n_single = n;
    const cudaError_t e = sort_launch(s, lay.sl, ws, scalars, sd, lay.K, offsets, entries, &launches);
    if (e != cudaSuccess) return record_error(e, "sort");
  }
  profile_mark(s, "sort");
  if (bases_ready) GM_CHECK(cudaStreamWaitEvent(s, bases_ready, 0));
  if (bases == nullptr) {
    uint4 *packed = (uint4 *)(ws + lay.o_packed);
    k_pack_ref<F><<<grid_for(n, 256), 256, 0, s>>>(packed, ref_points, n, 2 * H + 1, to_mont);
    GM_CHECK_LAUNCH("k_pack_ref");
    bases = packed;
    launches++;
    profile_mark(s, "pack");
  }
  acc_launch<F>(grid_for(lay.nthreads, ACC_THREADS), s, bases, entries, offsets, lay.K, lay.nthreads, buckets, head,
                tail, hk, tk);
  GM_CHECK_LAUNCH("k_accumulate");
  launches++;
  profile_mark(s, "accumulate");
  int rc = fixup_launch<F>(s, offsets, lay.K, lay.nthreads, buckets, head, tail, hk, tk, err, long_q, lay.long_cap,
                           &launches);
  if (rc) return rc;
  profile_mark(s, "fixup");

  // bucket reduction: leveled running sums, then a quad fan-in tree
  const int W = lay.dp.W;
  const xyzz_t<F> *src = nullptr;
  rc = reduce_launch<F>(s, lay.rl, buckets, offsets, ws, &src, &launches);
  if (rc) return rc;
  profile_mark(s, "reduce");
  // window combination: the serial Horner tail runs on the host (lower
  // latency per product) unless the stream is being captured into a graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GM_CHECK(cudaStreamIsCapturing(s, &cap));
  if (handoff && cap != cudaStreamCaptureStatusNone) {
    set_last_error("window-sum handoff while the stream is being captured");
    return GM_ERR_ARG;
  }
  if (handoff) {
    const size_t bytes = (size_t)W * sizeof(xyzz_t<F>);
    if (bytes > handoff->cap) {
      set_last_error("window-sum handoff buffer too small");
      return GM_ERR_ARG;
    }
    GM_CHECK(cudaMemcpyAsync(handoff->host, src, bytes, cudaMemcpyDeviceToHost, s));
    handoff->W = W;
    handoff->c = lay.dp.c;
  } else if (host_tail && cap == cudaStreamCaptureStatusNone) {
    rc = enqueue_host_tail(s, F::LIMBS == NL ? 1 : 2, src, W, lay.dp.c, out_proj);
    if (rc) return rc;
  } else {
    k_combine_quad<F><<<1, 32, 0, s>>>(src, 1, W, lay.dp.c, nullptr, out_proj);
    GM_CHECK_LAUNCH("k_combine_quad");
    launches++;
  }
  profile_mark(s, "combine");
  count_launches(launches);
  if (err_out) GM_CHECK(cudaMemcpyAsync(err_out, err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  return GM_OK;
}

// The whole pipeline with its workspace from the device's stream-ordered
// pool, released on s after the last kernel (also when an enqueue fails).
// c_override 0: the window width from the cost model.
template <class F>
int msm_launch(cudaStream_t s, int dev, const uint4 *bases, const uint64_t *ref_points, int to_mont,
               const uint64_t *scalars, int limbs, int64_t n, uint64_t *out_proj, int c_override,
               uint32_t *err_out, cudaEvent_t bases_ready, TailHandoff *handoff) {
  constexpr int H = F::LIMBS / 2;
  if (n == 0) {
    if (err_out) GM_CHECK(cudaMemsetAsync(err_out, 0, sizeof(uint32_t), s));
    GM_CHECK(cudaMemsetAsync(out_proj, 0, 3 * H * sizeof(uint64_t), s));
    return GM_OK;
  }
  const int c = c_override > 0 ? c_override : default_window(sizeof(typename F::T) == sizeof(fp_t) ? 1 : 2, n, limbs);
  MsmLayout<F> lay;
  int rc = msm_plan<F>(lay, dev, n, limbs, c, bases == nullptr, 0);
  if (rc) return rc;
  char *ws = nullptr;
  rc = pool_alloc(dev, s, lay.bytes, (void **)&ws);
  if (rc) return rc;
  rc = msm_run<F>(s, lay, ws, bases, ref_points, to_mont, scalars, out_proj, host_tail_enabled(), err_out,
                  bases_ready, handoff);
  const cudaError_t e = cudaFreeAsync(ws, s);
  if (rc) return rc;
  return e == cudaSuccess ? GM_OK : record_error(e, "cudaFreeAsync(workspace)");
}

}  // namespace gm
