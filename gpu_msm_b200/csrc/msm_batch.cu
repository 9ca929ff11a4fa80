// C-ABI of resident base tables and batched MSM plans (include/gpu_msm_b200.h,
// part 2).  The reference has neither: every reference MSM call copies its
// bases in and converts them again (rust-api/src/c_wrapper.cu:64-172).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/gpu_msm_b200.h"
#include "msm_batch.cuh"

namespace gm {
// heavy templates are instantiated once, in msm_g1.cu / msm_g2.cu
extern template int msm_launch<Fp>(cudaStream_t, int, const uint4 *, const uint64_t *, int, const uint64_t *, int,
                                   int64_t, uint64_t *, int, uint32_t *, cudaEvent_t, TailHandoff *);
extern template int msm_launch<Fp2>(cudaStream_t, int, const uint4 *, const uint64_t *, int, const uint64_t *, int,
                                    int64_t, uint64_t *, int, uint32_t *, cudaEvent_t, TailHandoff *);
extern template int batch_layouts<Fp>(BatchPlan &, int);
extern template int batch_layouts<Fp2>(BatchPlan &, int);
extern template int batch_run<Fp>(const BatchPlan &, cudaStream_t, const uint64_t *, uint64_t *);
extern template int batch_run<Fp2>(const BatchPlan &, cudaStream_t, const uint64_t *, uint64_t *);
extern template int window_table_launch<Fp>(cudaStream_t, const uint4 *, int64_t, int, int, uint4 *);
extern template int window_table_launch<Fp2>(cudaStream_t, const uint4 *, int64_t, int, int, uint4 *);
extern template int batch_queue_setup<Fp>(BatchPlan &);
extern template int batch_queue_setup<Fp2>(BatchPlan &);
}  // namespace gm

struct gm_bases {
  int group = 1;
  int dev = 0;
  int64_t n = 0;
  uint4 *packed = nullptr;  // owned, Rec<F>::U4 uint4 per point
  // fixed-base window tables (gm_bases_precompute): record w*n + i holds
  // 2^(c w) * point i, w < W
  struct WindowTable {
    int c = 0, W = 0;
    uint4 *table = nullptr;  // owned
  };
  std::vector<WindowTable> tables;

  const WindowTable *table_for(int c, int W) const {
    for (const auto &t : tables)
      if (t.c == c && t.W >= W) return &t;
    return nullptr;
  }
};

struct gm_batch_plan {
  gm::BatchPlan plan;
};

namespace {

void free_plan(gm_batch_plan *p) {
  for (auto &cp : p->plan.classes) {
    if (cp.ws) cudaFree(cp.ws);
    if (cp.desc) cudaFree(cp.desc);
    if (cp.stream) cudaStreamDestroy(cp.stream);
    if (cp.done) cudaEventDestroy(cp.done);
    if (cp.sorted) cudaEventDestroy(cp.sorted);
  }
  if (p->plan.fork) cudaEventDestroy(p->plan.fork);
  if (p->plan.acc_done) cudaEventDestroy(p->plan.acc_done);
  if (p->plan.acc_desc) cudaFree(p->plan.acc_desc);
  if (p->plan.queue_ctr) cudaFree(p->plan.queue_ctr);
  delete p;
}

// Validates the batch, groups MSMs by window width and computes each class's
// layout; d64[k] / idx[k] receive class k's descriptors
// (point_start | base_off | sc_off, and out_index | tile_first).
// tuning (optional): per MSM, the accumulation slices of its class in
// resident waves (tuning[2 i]: 1, 2 or 4; 0 = 1) and the pass-A sort tile in
// points per thread (tuning[2 i + 1]: 2, 4 or 8; 0 = 4); a class takes the
// values of its largest MSM.
int build_classes(const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes, const int64_t *base_offsets,
                  const int32_t *window_bits, gm::BatchPlan &plan, std::vector<std::vector<int64_t>> &d64,
                  std::vector<std::vector<int32_t>> &idx, const int32_t *tuning = nullptr) {
  if (!b || count <= 0 || !sizes || scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  int rc = gm::select_device((uint32_t)b->dev);
  if (rc) return rc;
  std::map<int, std::vector<int>> by_c;
  std::vector<int64_t> sc_row(count + 1, 0);
  for (int i = 0; i < count; i++) {
    const int64_t off = base_offsets ? base_offsets[i] : 0;
    if (sizes[i] <= 0 || off < 0 || off + sizes[i] > b->n) {
      gm::set_last_error("batch MSM outside the base table or empty");
      return gm::GM_ERR_ARG;
    }
    sc_row[i + 1] = sc_row[i] + sizes[i];
    int c = window_bits && window_bits[i] > 0 ? window_bits[i] : 0;
    if (c == 0 && !b->tables.empty()) {
      // with fixed-base tables an MSM costs ~10 products per (point, non-zero
      // window) plus 2 additions (28 products) per bucket of its single
      // bucket set; take the cheapest table
      double best = 0;
      for (const auto &t : b->tables) {
        if (t.W < gm::windows_for(t.c, scalar_limbs)) continue;
        const double cost = 10.0 * (double)sizes[i] * (64.0 * scalar_limbs / t.c) + 28.0 * (double)(1 << (t.c - 1));
        if (c == 0 || cost < best) {
          best = cost;
          c = t.c;
        }
      }
    }
    if (c == 0) c = gm::default_window(b->group, sizes[i], scalar_limbs);
    if (c < 2 || c > 20) {
      gm::set_last_error("window width out of range");
      return gm::GM_ERR_ARG;
    }
    by_c[c].push_back(i);
  }
  plan.group = b->group;
  plan.dev = b->dev;
  plan.limbs = scalar_limbs;
  plan.count = count;
  plan.bases = b->packed;
  plan.n_bases = b->n;
  plan.classes.clear();
  for (auto &kv : by_c) {
    gm::BatchClassPlan cp;
    cp.c = kv.first;
    cp.count = (int)kv.second.size();
    int largest = kv.second[0];
    for (int i : kv.second)
      if (sizes[i] > sizes[largest]) largest = i;
    if (tuning) {
      const int waves = tuning[2 * largest], ppt = tuning[2 * largest + 1];
      if (waves != 0 && waves != 1 && waves != 2 && waves != 4) {
        gm::set_last_error("batch tuning: slice waves must be 1, 2 or 4");
        return gm::GM_ERR_ARG;
      }
      if (ppt != 0 && ppt != 2 && ppt != 4 && ppt != 8) {
        gm::set_last_error("batch tuning: sort tile must be 2, 4 or 8 points per thread");
        return gm::GM_ERR_ARG;
      }
      cp.slice_waves = waves ? waves : 1;
      cp.sort_ppt = ppt ? ppt : gm::SA_PPT;
    }
    const int64_t tp = (int64_t)gm::SA_THREADS * cp.sort_ppt;
    for (int i : kv.second) {
      cp.P += sizes[i];
      cp.tilesA += (sizes[i] + tp - 1) / tp;
    }
    if (const auto *t = b->table_for(cp.c, gm::windows_for(cp.c, scalar_limbs))) {
      cp.pc_table = t->table;
      cp.pc_stride = b->n;
    }
    plan.classes.push_back(cp);
  }
  int sms = 0;
  rc = gm::device_sm_count(b->dev, &sms);
  if (rc) return rc;
  if (b->group == 1)
    gm::batch_layouts<gm::Fp>(plan, sms);
  else
    gm::batch_layouts<gm::Fp2>(plan, sms);
  d64.assign(plan.classes.size(), {});
  idx.assign(plan.classes.size(), {});
  size_t k = 0;
  for (auto &kv : by_c) {
    gm::BatchClassPlan &cp = plan.classes[k];
    if ((uint64_t)cp.P * cp.dp.W >= (1ull << 32)) {
      gm::set_last_error("batch class too large for 32-bit entry offsets");
      return gm::GM_ERR_ARG;
    }
    if (cp.tilesA >= (int64_t)INT32_MAX) {
      gm::set_last_error("batch class has too many sort tiles");
      return gm::GM_ERR_ARG;
    }
    std::vector<int64_t> &v = d64[k];
    v.assign(3 * (size_t)cp.count + 1, 0);
    // out_index[count] | tile_first[count + 1]
    idx[k].assign(2 * (size_t)cp.count + 1, 0);
    int64_t acc = 0;
    int32_t tiles = 0;
    for (int j = 0; j < cp.count; j++) {
      const int i = kv.second[j];
      v[j] = acc;
      acc += sizes[i];
      v[cp.count + 1 + j] = base_offsets ? base_offsets[i] : 0;
      v[2 * cp.count + 1 + j] = sc_row[i];
      idx[k][j] = i;
      idx[k][cp.count + j] = tiles;
      const int64_t tp = (int64_t)gm::SA_THREADS * cp.sort_ppt;
      tiles += (int32_t)((sizes[i] + tp - 1) / tp);
    }
    v[cp.count] = acc;
    idx[k][2 * (size_t)cp.count] = tiles;
    k++;
  }
  return gm::GM_OK;
}

}  // namespace

// Device bytes of a transient batch (descriptors and workspaces of every
// class, each 256-byte aligned): the figure gm_batch_workspace_bytes reports
// and gm_batch_run_ws requires.
static int64_t transient_bytes(const gm::BatchPlan &plan, const std::vector<std::vector<int64_t>> &d64,
                               const std::vector<std::vector<int32_t>> &idx) {
  int64_t bytes = 0;
  for (size_t k = 0; k < plan.classes.size(); k++)
    bytes += (int64_t)(plan.classes[k].ws_bytes + d64[k].size() * sizeof(int64_t) + idx[k].size() * sizeof(int32_t) +
                       512);
  return bytes;
}

extern "C" {

int gm_bases_create(uint32_t gpu_index, int group, const void *d_points, int64_t n, int points_montgomery,
                    gm_bases **out) {
  if (out == nullptr || (group != 1 && group != 2) || n <= 0 || n >= (int64_t(1) << 31) || d_points == nullptr)
    return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  auto *b = new (std::nothrow) gm_bases;
  if (!b) return gm::GM_ERR_ALLOC;
  b->group = group;
  b->dev = (int)gpu_index;
  b->n = n;
  const int u4 = group == 1 ? gm::Rec<gm::Fp>::U4 : gm::Rec<gm::Fp2>::U4;
  cudaError_t e = cudaMalloc(&b->packed, (size_t)n * u4 * sizeof(uint4));
  if (e != cudaSuccess) {
    delete b;
    gm::record_error(e, "cudaMalloc(bases)");
    return gm::GM_ERR_ALLOC;
  }
  const unsigned grid = (unsigned)((n + 255) / 256);
  const int to_mont = points_montgomery ? 0 : 1;
  if (group == 1)
    gm::k_pack_ref<gm::Fp><<<grid, 256>>>(b->packed, (const uint64_t *)d_points, n, 15, to_mont);
  else
    gm::k_pack_ref<gm::Fp2><<<grid, 256>>>(b->packed, (const uint64_t *)d_points, n, 29, to_mont);
  gm::count_launches(1);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaFree(b->packed);
    delete b;
    return gm::record_error(e, "k_pack_ref(bases)");
  }
  *out = b;
  return gm::GM_OK;
}

int gm_bases_destroy(gm_bases *b) {
  if (!b) return gm::GM_OK;
  cudaSetDevice(b->dev);
  cudaFree(b->packed);
  for (auto &t : b->tables) cudaFree(t.table);
  delete b;
  return gm::GM_OK;
}

int gm_bases_precompute(gm_bases *b, int window_bits, int scalar_limbs) {
  if (!b || window_bits < 2 || window_bits > 20 || scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS)
    return gm::GM_ERR_ARG;
  const int W = gm::windows_for(window_bits, scalar_limbs);
  if (b->table_for(window_bits, W)) return gm::GM_OK;
  if ((uint64_t)b->n * W >= (1ull << 31)) {
    gm::set_last_error("window table too large for 31-bit record indices");
    return gm::GM_ERR_ARG;
  }
  int rc = gm::select_device((uint32_t)b->dev);
  if (rc) return rc;
  const int u4 = b->group == 1 ? gm::Rec<gm::Fp>::U4 : gm::Rec<gm::Fp2>::U4;
  gm_bases::WindowTable t;
  t.c = window_bits;
  t.W = W;
  cudaError_t e = cudaMalloc(&t.table, (size_t)b->n * W * u4 * sizeof(uint4));
  if (e != cudaSuccess) {
    gm::record_error(e, "cudaMalloc(window table)");
    return gm::GM_ERR_ALLOC;
  }
  rc = b->group == 1 ? gm::window_table_launch<gm::Fp>(nullptr, b->packed, b->n, window_bits, W, t.table)
                     : gm::window_table_launch<gm::Fp2>(nullptr, b->packed, b->n, window_bits, W, t.table);
  if (rc == gm::GM_OK) {
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = gm::record_error(e, "k_window_table");
  }
  if (rc) {
    cudaFree(t.table);
    return rc;
  }
  b->tables.push_back(t);
  return gm::GM_OK;
}

int64_t gm_bases_count(const gm_bases *b) { return b ? b->n : 0; }

int gm_msm_resident(gm_stream_t stream, const gm_bases *b, int64_t base_offset, int n, const uint64_t *d_scalars,
                    int scalar_limbs, void *d_result, int window_bits) {
  if (!b || d_result == nullptr || n < 0 || base_offset < 0 || base_offset + n > b->n ||
      (n > 0 && d_scalars == nullptr))
    return gm::GM_ERR_ARG;
  int rc = gm::select_device((uint32_t)b->dev);
  if (rc) return rc;
  if (!b->tables.empty() && n > 0) {
    // fixed-base tables: a batch of one (single bucket set, no window doublings)
    const int64_t size = n;
    const int32_t wb = window_bits;
    return gm_batch_run(stream, b, scalar_limbs, 1, &size, &base_offset, window_bits > 0 ? &wb : nullptr, d_scalars,
                        d_result);
  }
  if (b->group == 1)
    return gm::msm_launch<gm::Fp>((cudaStream_t)stream, b->dev, b->packed + base_offset * gm::Rec<gm::Fp>::U4, nullptr,
                                  0, d_scalars, scalar_limbs, n, (uint64_t *)d_result, window_bits, nullptr);
  return gm::msm_launch<gm::Fp2>((cudaStream_t)stream, b->dev, b->packed + base_offset * gm::Rec<gm::Fp2>::U4, nullptr,
                                 0, d_scalars, scalar_limbs, n, (uint64_t *)d_result, window_bits, nullptr);
}

int gm_batch_plan_create(const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                         const int64_t *base_offsets, const int32_t *window_bits, gm_batch_plan **out) {
  return gm_batch_plan_create_tuned(b, scalar_limbs, count, sizes, base_offsets, window_bits, nullptr, out);
}

int gm_batch_plan_create_tuned(const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                               const int64_t *base_offsets, const int32_t *window_bits, const int32_t *tuning,
                               gm_batch_plan **out) {
  if (!b || !out) return gm::GM_ERR_ARG;
  auto *p = new (std::nothrow) gm_batch_plan;
  if (!p) return gm::GM_ERR_ALLOC;
  std::vector<std::vector<int64_t>> d64;
  std::vector<std::vector<int32_t>> idx;
  int rc = build_classes(b, scalar_limbs, count, sizes, base_offsets, window_bits, p->plan, d64, idx, tuning);
  if (rc) {
    delete p;
    return rc;
  }
  gm::BatchPlan &plan = p->plan;
  for (size_t k = 0; k < plan.classes.size(); k++) {
    gm::BatchClassPlan &cp = plan.classes[k];
    const size_t desc_bytes = d64[k].size() * sizeof(int64_t) + idx[k].size() * sizeof(int32_t);
    cudaError_t e = cudaMalloc(&cp.desc, desc_bytes);
    if (e == cudaSuccess) e = cudaMemcpy(cp.desc, d64[k].data(), d64[k].size() * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(cp.desc + d64[k].size() * sizeof(int64_t), idx[k].data(), idx[k].size() * sizeof(int32_t),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&cp.ws, cp.ws_bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cp.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&cp.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&cp.sorted, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      free_plan(p);
      gm::record_error(e, "batch plan allocation");
      return gm::GM_ERR_ALLOC;
    }
    plan.bytes += cp.ws_bytes + desc_bytes;
  }
  cudaError_t e = cudaEventCreateWithFlags(&plan.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&plan.acc_done, cudaEventDisableTiming);
  // descriptors of the queued accumulation (used when the plan's mode is set)
  const size_t desc_bytes = plan.classes.size() *
                            (plan.group == 1 ? sizeof(gm::AccClass<gm::Fp>) : sizeof(gm::AccClass<gm::Fp2>));
  if (e == cudaSuccess) e = cudaMalloc(&plan.acc_desc, desc_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&plan.queue_ctr, sizeof(uint32_t));
  if (e != cudaSuccess) {
    free_plan(p);
    return gm::record_error(e, "batch plan events / queue");
  }
  rc = plan.group == 1 ? gm::batch_queue_setup<gm::Fp>(plan) : gm::batch_queue_setup<gm::Fp2>(plan);
  if (rc) {
    free_plan(p);
    return rc;
  }
  plan.bytes += desc_bytes + sizeof(uint32_t);
  *out = p;
  return gm::GM_OK;
}

int gm_batch_plan_set_queue(gm_batch_plan *p, int on) {
  if (!p) return gm::GM_ERR_ARG;
  p->plan.queue = on != 0;
  return gm::GM_OK;
}

int64_t gm_batch_workspace_bytes(const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                                 const int32_t *window_bits) {
  gm::BatchPlan plan;
  std::vector<std::vector<int64_t>> d64;
  std::vector<std::vector<int32_t>> idx;
  if (build_classes(b, scalar_limbs, count, sizes, nullptr, window_bits, plan, d64, idx)) return -1;
  return transient_bytes(plan, d64, idx);
}

// gm_batch_run / gm_batch_run_ws: ws == nullptr takes the workspace from the
// stream-ordered pool for this run; otherwise the caller's ws_bytes at ws.
static int batch_run_once(gm_stream_t stream, const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                   const int64_t *base_offsets, const int32_t *window_bits, const uint64_t *d_scalars,
                   void *d_results, void *ws, size_t ws_bytes) {
  if (!d_scalars || !d_results) return gm::GM_ERR_ARG;
  gm::BatchPlan plan;
  std::vector<std::vector<int64_t>> d64;
  std::vector<std::vector<int32_t>> idx;
  int rc = build_classes(b, scalar_limbs, count, sizes, base_offsets, window_bits, plan, d64, idx);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // one stream-ordered allocation: every class's descriptors first (so they
  // can be staged contiguously), then the workspaces
  std::vector<size_t> off_desc(plan.classes.size()), off_ws(plan.classes.size());
  size_t total = 0;
  for (size_t k = 0; k < plan.classes.size(); k++) {
    off_desc[k] = total;
    total += (d64[k].size() * sizeof(int64_t) + idx[k].size() * sizeof(int32_t) + 255) / 256 * 256;
  }
  const size_t desc_total = total;
  for (size_t k = 0; k < plan.classes.size(); k++) {
    off_ws[k] = total;
    total += (plan.classes[k].ws_bytes + 255) / 256 * 256;
  }
  char *mem = nullptr;
  if (ws) {
    if (total > ws_bytes || (size_t)transient_bytes(plan, d64, idx) > ws_bytes ||
        (reinterpret_cast<uintptr_t>(ws) & 255u)) {
      gm::set_last_error("batch workspace too small or not 256-byte aligned");
      return gm::GM_ERR_ARG;
    }
    mem = static_cast<char *>(ws);
  } else {
    rc = gm::pool_alloc(plan.dev, s, total, (void **)&mem);
    if (rc) return rc;
  }
  // descriptors go through one pinned slot (an asynchronous copy from pageable
  // memory would first wait for the stream), released in stream order
  void *slot = nullptr;
  const bool pinned = desc_total <= gm::PINNED_SLOT_BYTES && gm::pinned_acquire(&slot) == gm::GM_OK;
  for (size_t k = 0; k < plan.classes.size(); k++) {
    gm::BatchClassPlan &cp = plan.classes[k];
    cp.desc = mem + off_desc[k];
    cp.ws = mem + off_ws[k];
    const size_t n64 = d64[k].size() * sizeof(int64_t), n32 = idx[k].size() * sizeof(int32_t);
    cudaError_t e;
    if (pinned) {
      char *h = static_cast<char *>(slot) + off_desc[k];
      memcpy(h, d64[k].data(), n64);
      memcpy(h + n64, idx[k].data(), n32);
      e = cudaMemcpyAsync(cp.desc, h, n64 + n32, cudaMemcpyHostToDevice, s);
    } else {
      e = cudaMemcpyAsync(cp.desc, d64[k].data(), n64, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(cp.desc + n64, idx[k].data(), n32, cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) {
      if (pinned) gm::enqueue_pinned_release(s, slot);
      if (!ws) cudaFreeAsync(mem, s);
      return gm::record_error(e, "batch descriptors");
    }
  }
  if (pinned) gm::enqueue_pinned_release(s, slot);
  rc = plan.group == 1 ? gm::batch_run<gm::Fp>(plan, s, d_scalars, (uint64_t *)d_results)
                       : gm::batch_run<gm::Fp2>(plan, s, d_scalars, (uint64_t *)d_results);
  if (!ws) cudaFreeAsync(mem, s);
  return rc;
}

int gm_batch_run(gm_stream_t stream, const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                 const int64_t *base_offsets, const int32_t *window_bits, const uint64_t *d_scalars,
                 void *d_results) {
  return batch_run_once(stream, b, scalar_limbs, count, sizes, base_offsets, window_bits, d_scalars, d_results,
                        nullptr, 0);
}

int gm_batch_run_ws(gm_stream_t stream, const gm_bases *b, int scalar_limbs, int count, const int64_t *sizes,
                    const int64_t *base_offsets, const int32_t *window_bits, const uint64_t *d_scalars,
                    void *d_results, void *d_workspace, int64_t workspace_bytes) {
  if (!d_workspace || workspace_bytes <= 0) return gm::GM_ERR_ARG;
  return batch_run_once(stream, b, scalar_limbs, count, sizes, base_offsets, window_bits, d_scalars, d_results,
                        d_workspace, (size_t)workspace_bytes);
}

int gm_batch_plan_run(gm_batch_plan *p, gm_stream_t stream, const uint64_t *d_scalars, void *d_results) {
  if (!p || !d_scalars || !d_results) return gm::GM_ERR_ARG;
  int rc = gm::select_device((uint32_t)p->plan.dev);
  if (rc) return rc;
  if (p->plan.group == 1) return gm::batch_run<gm::Fp>(p->plan, (cudaStream_t)stream, d_scalars, (uint64_t *)d_results);
  return gm::batch_run<gm::Fp2>(p->plan, (cudaStream_t)stream, d_scalars, (uint64_t *)d_results);
}

int gm_batch_plan_destroy(gm_batch_plan *p) {
  if (!p) return gm::GM_OK;
  cudaSetDevice(p->plan.dev);
  cudaDeviceSynchronize();
  free_plan(p);
  return gm::GM_OK;
}

int64_t gm_batch_plan_bytes(const gm_batch_plan *p) { return p ? (int64_t)p->plan.bytes : 0; }

int gm_batch_plan_classes(const gm_batch_plan *p, int32_t *window_bits, int32_t *counts, int max) {
  if (!p) return 0;
  int k = 0;
  for (const auto &cp : p->plan.classes) {
    if (k < max) {
      if (window_bits) window_bits[k] = cp.c;
      if (counts) counts[k] = cp.count;
    }
    k++;
  }
  return k;
}

}  // extern "C"
