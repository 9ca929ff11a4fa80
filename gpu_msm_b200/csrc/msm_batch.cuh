// Batched MSM engine: many independent MSMs of uneven size over one resident
// base table, executed as one flattened pipeline per window-width class.
//
// A plan fixes the batch's shape (sizes, base offsets, window width per MSM),
// groups the MSMs into classes of equal window width, uploads the per-MSM
// descriptors and allocates every workspace once.  Running the plan only
// enqueues kernels and memsets: each class on its own stream, forked from and
// joined back to the caller's stream with events, so a run can be captured
// into a CUDA graph and replayed with new scalars in the same buffer.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "msm_host.cuh"

namespace gm {

struct BatchClassPlan {
  int c = 0;
  DigitParams dp{};
  int count = 0;        // MSMs in this class
  int64_t P = 0;        // points in this class
  int64_t K = 0, nthreads = 0;
  int64_t tilesA = 0;   // pass-A sort tiles (SA_TP points, one MSM each)
  SortLayout sl;
  RedLayout rl;
  int64_t long_cap = 0;
  // fixed-base window table (precomputed mode): record w*pc_stride + base
  const uint4 *pc_table = nullptr;
  int64_t pc_stride = 0;
  size_t o_offsets = 0, o_entries = 0, o_buckets = 0, o_head = 0, o_tail = 0, o_hk = 0, o_tk = 0, o_longq = 0,
         o_err = 0;
  size_t ws_bytes = 0;
  char *ws = nullptr;       // workspace (owned)
  // descriptors (owned): int64 point_start[count+1] | base_off[count] |
  // sc_off[count], then int32 out_index[count] | tile_first[count+1]
  char *desc = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

struct BatchPlan {
  int group = 1, dev = 0, limbs = 1, count = 0;
  const uint4 *bases = nullptr;
  int64_t n_bases = 0;
  std::vector<BatchClassPlan> classes;
  cudaEvent_t fork = nullptr;
  size_t bytes = 0;
};

// Workspace layout of one class (same parts as a single MSM, K over all the
// class's MSMs, no base packing).
template <class F>
void batch_class_layout(BatchClassPlan &cp, int limbs, int sms, int dev) {
  cp.dp.c = cp.c;
  cp.dp.W = windows_for(cp.c, limbs);
  cp.dp.B = 1 << (cp.c - 1);
  cp.dp.limbs = limbs;
  // precomputed mode: one bucket set per MSM (no window index in the key)
  const int64_t groups = (int64_t)cp.count * (cp.pc_stride ? 1 : cp.dp.W);
  cp.K = groups * cp.dp.B;
  cp.nthreads = (int64_t)sms * acc_blocks_per_sm<F>(dev) * ACC_THREADS;
  const int64_t max_entries = cp.P * cp.dp.W;
  if (cp.nthreads > max_entries) cp.nthreads = std::max<int64_t>(1, (max_entries + 127) / 128 * 128);
  Carve cv;
  cp.o_offsets = cv.take<uint32_t>(cp.K + 1);
  cp.o_entries = cv.take<uint32_t>((size_t)std::max<int64_t>(1, max_entries));
  cp.sl.plan(cp.dp, cp.count, cp.P, cp.tilesA, cp.pc_stride != 0, cv);
  cp.o_buckets = cv.take<xyzz_t<F>>(cp.K);
  cp.o_head = cv.take<xyzz_t<F>>(cp.nthreads);
  cp.o_tail = cv.take<xyzz_t<F>>(cp.nthreads);
  cp.o_hk = cv.take<int32_t>(cp.nthreads);
  cp.o_tk = cv.take<int32_t>(cp.nthreads);
  cp.rl.plan<F>(groups, cp.dp.B, (int64_t)sms * level0_blocks_per_sm<F>(dev) * 128, cv, coop_wave_threads<F>(dev, sms));
  cp.rl.sms = sms;
  cp.rl.dev = dev;
  cp.long_cap = cp.nthreads / FIX_SHORT + 1;
  cp.o_longq = cv.take<int32_t>((size_t)(1 + cp.long_cap));
  cp.o_err = cv.take<uint32_t>(4);
  cp.ws_bytes = cv.off;
}

// Enqueue one class's pipeline on `s`.
template <class F>
int batch_class_run(const BatchPlan &plan, const BatchClassPlan &cp, cudaStream_t s, const uint64_t *scalars,
                    uint64_t *results) {
  if (cp.count == 0) return GM_OK;
  char *ws = cp.ws;
  auto *offsets = (uint32_t *)(ws + cp.o_offsets);
  auto *entries = (uint32_t *)(ws + cp.o_entries);
  auto *buckets = (xyzz_t<F> *)(ws + cp.o_buckets);
  auto *head = (xyzz_t<F> *)(ws + cp.o_head);
  auto *tail = (xyzz_t<F> *)(ws + cp.o_tail);
  auto *hk = (int32_t *)(ws + cp.o_hk);
  auto *tk = (int32_t *)(ws + cp.o_tk);
  auto *err = (uint32_t *)(ws + cp.o_err);
  auto *long_q = (int32_t *)(ws + cp.o_longq);
  SortDesc sd;
  sd.point_start = (const int64_t *)cp.desc;
  sd.base_off = sd.point_start + cp.count + 1;
  sd.sc_off = sd.base_off + cp.count;
  sd.count = cp.count;
  sd.pc_stride = cp.pc_stride;
  const int32_t *out_index = (const int32_t *)(sd.sc_off + cp.count);
  sd.tile_first = out_index + cp.count;

  int launches = 0;
  GM_CHECK(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  GM_CHECK(cudaMemsetAsync(long_q, 0, sizeof(int32_t), s));
  {
    const cudaError_t e = sort_launch(s, cp.sl, ws, scalars, sd, cp.K, offsets, entries, &launches);
    if (e != cudaSuccess) return record_error(e, "batch sort");
  }
  acc_launch<F>(grid_for(cp.nthreads, ACC_THREADS), s, cp.pc_table ? cp.pc_table : plan.bases, entries,
                offsets, cp.K, cp.nthreads, buckets, head, tail, hk, tk);
  GM_CHECK_LAUNCH("k_accumulate");
  launches++;
  int rc = fixup_launch<F>(s, offsets, cp.K, cp.nthreads, buckets, head, tail, hk, tk, err, long_q, cp.long_cap,
                           &launches);
  if (rc) return rc;
  const xyzz_t<F> *src = nullptr;
  rc = reduce_launch<F>(s, cp.rl, buckets, offsets, ws, &src, &launches);
  if (rc) return rc;
  // precomputed mode: one window per MSM, so the combination is a conversion
  k_combine_quad<F><<<grid_for((int64_t)Coop<F>::LANES * cp.count, 128), 128, 0, s>>>(src, cp.count, cp.pc_stride ? 1 : cp.dp.W,
                                                                          cp.c, out_index, results);
  GM_CHECK_LAUNCH("k_combine_quad");
  launches++;
  count_launches(launches);
  return GM_OK;
}

// Builds the fixed-base window table of n packed points: W windows of c bits.
template <class F>
int window_table_launch(cudaStream_t s, const uint4 *packed, int64_t n, int c, int W, uint4 *table) {
  k_window_table<F><<<grid_for(n, 128), 128, 0, s>>>(packed, n, c, W, table);
  GM_CHECK_LAUNCH("k_window_table");
  count_launches(1);
  return GM_OK;
}

template <class F>
int batch_layouts(BatchPlan &plan, int sms) {
  for (auto &cp : plan.classes) batch_class_layout<F>(cp, plan.limbs, sms, plan.dev);
  return GM_OK;
}

// Fork the classes onto their streams and join them back into `s` (plans
// with their own streams), or run them in order on `s`.
template <class F>
int batch_run(const BatchPlan &plan, cudaStream_t s, const uint64_t *scalars, uint64_t *results) {
  if (plan.classes.size() == 1 || plan.fork == nullptr) {
    // one class, or a transient plan without its own streams: in order on s
    for (const auto &cp : plan.classes) {
      const int rc = batch_class_run<F>(plan, cp, s, scalars, results);
      if (rc) return rc;
    }
    return GM_OK;
  }
  GM_CHECK(cudaEventRecord(plan.fork, s));
  for (const auto &cp : plan.classes) {
    GM_CHECK(cudaStreamWaitEvent(cp.stream, plan.fork, 0));
    const int rc = batch_class_run<F>(plan, cp, cp.stream, scalars, results);
    if (rc) return rc;
    GM_CHECK(cudaEventRecord(cp.done, cp.stream));
    GM_CHECK(cudaStreamWaitEvent(s, cp.done, 0));
  }
  return GM_OK;
}

}  // namespace gm
