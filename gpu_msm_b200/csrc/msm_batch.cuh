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
  int64_t tilesA = 0;   // pass-A sort tiles (SA_THREADS * sort_ppt points, one MSM each)
  int slice_waves = 1;  // accumulation slices: this many resident waves of threads
  int sort_ppt = SA_PPT;  // pass-A sort tile: points per thread (2, 4 or 8)
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
  cudaEvent_t sorted = nullptr;  // queued accumulation: this class's sort has run
};

struct BatchPlan {
  int group = 1, dev = 0, limbs = 1, count = 0;
  const uint4 *bases = nullptr;
  int64_t n_bases = 0;
  std::vector<BatchClassPlan> classes;
  cudaEvent_t fork = nullptr;
  size_t bytes = 0;
  // Accumulation mode of plans: true (default) = every class's accumulation
  // in one persistent launch over a device work queue (k_accumulate_queue)
  // between the classes' sorts and their fix-ups; false = one pipeline per
  // class on its own stream, every kernel of a class a full-GPU launch.
  // The 512-MSM batch (2^8..2^16 points, 2^16-point table) measured 145.3 ms
  // queued against 148.5-149.7 ms per class on B200, and 97.1 against
  // 97.4 ms with fixed-base window tables.  Transient batches
  // (gm_batch_run) run their classes in order on the caller's stream.
  bool queue = true;
  char *acc_desc = nullptr;      // AccClass<F>[classes] (owned)
  uint32_t *queue_ctr = nullptr; // work-queue counter (owned)
  int64_t queue_items = 0;
  cudaEvent_t acc_done = nullptr;
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
  cp.nthreads = (int64_t)sms * acc_blocks_per_sm<F>(dev) * ACC_THREADS * cp.slice_waves;
  const int64_t max_entries = cp.P * cp.dp.W;
  if (cp.nthreads > max_entries) cp.nthreads = std::max<int64_t>(1, (max_entries + 127) / 128 * 128);
  Carve cv;
  cp.o_offsets = cv.take<uint32_t>(cp.K + 1);
  cp.o_entries = cv.take<uint32_t>((size_t)std::max<int64_t>(1, max_entries));
  cp.sl.plan(cp.dp, cp.count, cp.P, cp.tilesA, cp.pc_stride != 0, cv, cp.sort_ppt);
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

// Pointers into one class's workspace.
template <class F>
struct ClassBufs {
  uint32_t *offsets, *entries, *err;
  int32_t *hk, *tk, *long_q;
  xyzz_t<F> *buckets, *head, *tail;
  SortDesc sd;
  const int32_t *out_index;
  ClassBufs(const BatchClassPlan &cp) {
    char *ws = cp.ws;
    offsets = (uint32_t *)(ws + cp.o_offsets);
    entries = (uint32_t *)(ws + cp.o_entries);
    buckets = (xyzz_t<F> *)(ws + cp.o_buckets);
    head = (xyzz_t<F> *)(ws + cp.o_head);
    tail = (xyzz_t<F> *)(ws + cp.o_tail);
    hk = (int32_t *)(ws + cp.o_hk);
    tk = (int32_t *)(ws + cp.o_tk);
    err = (uint32_t *)(ws + cp.o_err);
    long_q = (int32_t *)(ws + cp.o_longq);
    sd.point_start = (const int64_t *)cp.desc;
    sd.base_off = sd.point_start + cp.count + 1;
    sd.sc_off = sd.base_off + cp.count;
    sd.count = cp.count;
    sd.pc_stride = cp.pc_stride;
    out_index = (const int32_t *)(sd.sc_off + cp.count);
    sd.tile_first = out_index + cp.count;
  }
};

// One class, first part: flags cleared, entries sorted.
template <class F>
int batch_class_sort(const BatchClassPlan &cp, cudaStream_t s, const uint64_t *scalars, int *launches) {
  ClassBufs<F> cb(cp);
  GM_CHECK(cudaMemsetAsync(cb.err, 0, sizeof(uint32_t), s));
  GM_CHECK(cudaMemsetAsync(cb.long_q, 0, sizeof(int32_t), s));
  const cudaError_t e = sort_launch(s, cp.sl, cp.ws, scalars, cb.sd, cp.K, cb.offsets, cb.entries, launches);
  if (e != cudaSuccess) return record_error(e, "batch sort");
  return GM_OK;
}

// One class, last part (after its accumulation): fix-up, reduction, and the
// window combination into the class's result slots.
template <class F>
int batch_class_finish(const BatchClassPlan &cp, cudaStream_t s, uint64_t *results, int *launches) {
  ClassBufs<F> cb(cp);
  int rc = fixup_launch<F>(s, cb.offsets, cp.K, cp.nthreads, cb.buckets, cb.head, cb.tail, cb.hk, cb.tk, cb.err,
                           cb.long_q, cp.long_cap, launches);
  if (rc) return rc;
  const xyzz_t<F> *src = nullptr;
  rc = reduce_launch<F>(s, cp.rl, cb.buckets, cb.offsets, cp.ws, &src, launches);
  if (rc) return rc;
  // precomputed mode: one window per MSM, so the combination is a conversion
  k_combine_quad<F><<<grid_for((int64_t)Coop<F>::LANES * cp.count, 128), 128, 0, s>>>(
      src, cp.count, cp.pc_stride ? 1 : cp.dp.W, cp.c, cb.out_index, results);
  GM_CHECK_LAUNCH("k_combine_quad");
  (*launches)++;
  return GM_OK;
}

// Enqueue one class's whole pipeline on `s`.
template <class F>
int batch_class_run(const BatchPlan &plan, const BatchClassPlan &cp, cudaStream_t s, const uint64_t *scalars,
                    uint64_t *results) {
  if (cp.count == 0) return GM_OK;
  int launches = 0;
  int rc = batch_class_sort<F>(cp, s, scalars, &launches);
  if (rc) return rc;
  ClassBufs<F> cb(cp);
  acc_launch<F>(grid_for(cp.nthreads, ACC_THREADS), s, cp.pc_table ? cp.pc_table : plan.bases, cb.entries,
                cb.offsets, cp.K, cp.nthreads, cb.buckets, cb.head, cb.tail, cb.hk, cb.tk);
  GM_CHECK_LAUNCH("k_accumulate");
  launches++;
  rc = batch_class_finish<F>(cp, s, results, &launches);
  count_launches(launches);
  return rc;
}

// Device descriptors of the queued accumulation (plans with their own
// streams): one AccClass per class, written into plan.acc_desc.
template <class F>
int batch_queue_setup(BatchPlan &plan) {
  std::vector<AccClass<F>> h(plan.classes.size());
  int64_t items = 0;
  for (size_t k = 0; k < plan.classes.size(); k++) {
    const BatchClassPlan &cp = plan.classes[k];
    ClassBufs<F> cb(cp);
    h[k] = AccClass<F>{cp.pc_table ? cp.pc_table : plan.bases, cb.entries, cb.offsets, cp.K, cp.nthreads,
                       cb.buckets, cb.head, cb.tail, cb.hk, cb.tk, items};
    items += cp.nthreads / 32;  // nthreads is a multiple of 128
  }
  plan.queue_items = items;
  GM_CHECK(cudaMemcpy(plan.acc_desc, h.data(), h.size() * sizeof(AccClass<F>), cudaMemcpyHostToDevice));
  return GM_OK;
}

// The queued flow: every class sorts on its stream; s joins them, runs the
// accumulation of all classes in one persistent launch, and forks the
// classes again for their fix-ups, reductions and combinations.
template <class F>
int batch_run_queued(const BatchPlan &plan, cudaStream_t s, const uint64_t *scalars, uint64_t *results) {
  int launches = 0;
  GM_CHECK(cudaEventRecord(plan.fork, s));
  for (const auto &cp : plan.classes) {
    GM_CHECK(cudaStreamWaitEvent(cp.stream, plan.fork, 0));
    const int rc = batch_class_sort<F>(cp, cp.stream, scalars, &launches);
    if (rc) return rc;
    GM_CHECK(cudaEventRecord(cp.sorted, cp.stream));
    GM_CHECK(cudaStreamWaitEvent(s, cp.sorted, 0));
  }
  GM_CHECK(cudaMemsetAsync(plan.queue_ctr, 0, sizeof(uint32_t), s));
  int dev = 0, sms = 0;
  GM_CHECK(cudaGetDevice(&dev));
  int rc = device_sm_count(dev, &sms);
  if (rc) return rc;
  const AccOccupancy occ = acc_occupancy<F>(dev, 1);
  k_accumulate_queue<F><<<(unsigned)(sms * occ.blocks), ACC_THREADS, occ.smem, s>>>(
      (const AccClass<F> *)plan.acc_desc, (int)plan.classes.size(), plan.queue_items, plan.queue_ctr);
  GM_CHECK_LAUNCH("k_accumulate_queue");
  launches++;
  GM_CHECK(cudaEventRecord(plan.acc_done, s));
  for (const auto &cp : plan.classes) {
    GM_CHECK(cudaStreamWaitEvent(cp.stream, plan.acc_done, 0));
    rc = batch_class_finish<F>(cp, cp.stream, results, &launches);
    if (rc) return rc;
    GM_CHECK(cudaEventRecord(cp.done, cp.stream));
    GM_CHECK(cudaStreamWaitEvent(s, cp.done, 0));
  }
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
  if (plan.queue && plan.acc_desc) return batch_run_queued<F>(plan, s, scalars, results);
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
