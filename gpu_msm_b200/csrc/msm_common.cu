// Host side of the MSM engine shared by both groups: error bookkeeping,
// per-device state and memory pool, window selection.
//
// Replaces the reference's MSM drivers (pdroalves/gpu_msm src/curve.cu:2538-2826)
// and C wrappers (rust-api/src/c_wrapper.cu).  Unlike the reference, which
// copies 16 buckets to the host and blocks three times per window, the whole
// MSM here is one asynchronous launch sequence on the caller's stream with no
// host round trip; workspace comes from a per-device stream-ordered memory
// pool so concurrent calls on different streams never share scratch.
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gpu_msm_b200.h"
#include "host_arith.h"
#include "msm_engine.h"

namespace gm {

// ---------------------------------------------------------------------------
// error bookkeeping
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error = "";

int record_error(cudaError_t e, const char *where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return GM_ERR_CUDA;
}

const char *last_error() { return g_last_error.c_str(); }

void set_last_error(const char *msg) { g_last_error = msg; }

#define GM_CHECK(call)                                                  \
  do {                                                                  \
    cudaError_t _e = (call);                                            \
    if (_e != cudaSuccess) return record_error(_e, #call);              \
  } while (0)

#define GM_CHECK_LAUNCH(where)                                          \
  do {                                                                  \
    cudaError_t _e = cudaGetLastError();                                \
    if (_e != cudaSuccess) return record_error(_e, where);              \
  } while (0)

// ---------------------------------------------------------------------------
// per-device state: SM count and a stream-ordered pool that keeps memory
// cached between calls (release threshold = unlimited)
// ---------------------------------------------------------------------------
struct DeviceState {
  int sms = 0;
  cudaMemPool_t pool = nullptr;
};

static std::mutex g_dev_mu;
static std::map<int, DeviceState> g_dev;

int device_state(int dev, DeviceState **out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  auto it = g_dev.find(dev);
  if (it == g_dev.end()) {
    DeviceState st;
    GM_CHECK(cudaDeviceGetAttribute(&st.sms, cudaDevAttrMultiProcessorCount, dev));
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    GM_CHECK(cudaMemPoolCreate(&st.pool, &props));
    uint64_t thr = UINT64_MAX;
    GM_CHECK(cudaMemPoolSetAttribute(st.pool, cudaMemPoolAttrReleaseThreshold, &thr));
    it = g_dev.emplace(dev, st).first;
  }
  *out = &it->second;
  return GM_OK;
}

// ---------------------------------------------------------------------------
// phase profiling (CUDA events on the launching stream) and launch counting,
// per host thread
// ---------------------------------------------------------------------------
struct PhaseMark {
  const char *name;
  cudaEvent_t ev;
};
static thread_local bool g_prof_on = false;
static thread_local std::vector<PhaseMark> g_marks;
static thread_local std::vector<std::pair<std::string, float>> g_phase_ms;
static thread_local int64_t g_launches = 0;

void profile_enable(bool on) { g_prof_on = on; }
bool profile_enabled() { return g_prof_on; }

void profile_mark(cudaStream_t s, const char *name) {
  if (!g_prof_on) return;
  PhaseMark m{name, nullptr};
  if (cudaEventCreate(&m.ev) != cudaSuccess) return;
  cudaEventRecord(m.ev, s);
  g_marks.push_back(m);
}

// Closes the marks of one call: consecutive marks delimit phases.
void profile_end_call() {
  if (!g_prof_on) return;
  for (size_t i = 1; i < g_marks.size(); i++) {
    float ms = 0.f;
    cudaEventSynchronize(g_marks[i].ev);
    cudaEventElapsedTime(&ms, g_marks[i - 1].ev, g_marks[i].ev);
    g_phase_ms.emplace_back(g_marks[i].name, ms);
  }
  for (auto &m : g_marks) cudaEventDestroy(m.ev);
  g_marks.clear();
}

int profile_collect(char *names, int names_len, float *ms, int max) {
  profile_end_call();
  int n = 0;
  std::string joined;
  for (auto &p : g_phase_ms) {
    if (n < max) {
      ms[n] = p.second;
      if (!joined.empty()) joined += ",";
      joined += p.first;
    }
    n++;
  }
  if (names && names_len > 0) {
    strncpy(names, joined.c_str(), names_len - 1);
    names[names_len - 1] = 0;
  }
  g_phase_ms.clear();
  return n < max ? n : max;
}

void count_launches(int k) { g_launches += k; }
int64_t launches_and_reset() {
  const int64_t v = g_launches;
  g_launches = 0;
  return v;
}

// ---------------------------------------------------------------------------
// host tail: pinned slots and stream-ordered host functions
// ---------------------------------------------------------------------------
constexpr size_t TAIL_SLOT_BYTES = PINNED_SLOT_BYTES;  // >= 257 windows x 448 B + 336 B
static std::mutex g_pin_mu;
static std::vector<void *> g_pin_free;
// Slots whose last copy is still pending: returned to the free list once
// their event has completed.  A host function per release would cost a
// driver round trip (~0.2 ms of stream time on B200 boxes) for nothing.
struct PendingSlot {
  void *slot;
  cudaEvent_t ev;
  int dev;
};
static std::vector<PendingSlot> g_pin_pending;
static std::map<int, std::vector<cudaEvent_t>> g_free_events;  // per device
static bool g_host_tail = true;

bool host_tail_enabled() { return g_host_tail; }
void set_host_tail_enabled(bool on) { g_host_tail = on; }

// caller holds g_pin_mu
static void reclaim_completed_slots() {
  for (size_t i = 0; i < g_pin_pending.size();) {
    if (cudaEventQuery(g_pin_pending[i].ev) == cudaSuccess) {
      g_pin_free.push_back(g_pin_pending[i].slot);
      g_free_events[g_pin_pending[i].dev].push_back(g_pin_pending[i].ev);
      g_pin_pending[i] = g_pin_pending.back();
      g_pin_pending.pop_back();
    } else {
      i++;
    }
  }
}

int pinned_acquire(void **p) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) reclaim_completed_slots();
    if (!g_pin_free.empty()) {
      *p = g_pin_free.back();
      g_pin_free.pop_back();
      return GM_OK;
    }
  }
  cudaError_t e = cudaMallocHost(p, PINNED_SLOT_BYTES);
  if (e != cudaSuccess) return record_error(e, "cudaMallocHost(tail slot)");
  return GM_OK;
}

void pinned_release(void *p) {
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.push_back(p);
}

// The slot returns to the pool once the work enqueued on s so far has run.
int enqueue_pinned_release(cudaStream_t s, void *slot) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return record_error(e, "cudaGetDevice");
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto &fe = g_free_events[dev];
    if (!fe.empty()) {
      ev = fe.back();
      fe.pop_back();
    }
  }
  if (ev == nullptr) {
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    // without an event the slot stays with the stream's pending work: leak it
    // rather than hand it out again while a copy may still use it
    if (e != cudaSuccess) return record_error(e, "cudaEventCreate(slot)");
  }
  e = cudaEventRecord(ev, s);
  if (e != cudaSuccess) return record_error(e, "cudaEventRecord(slot)");
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_pending.push_back(PendingSlot{slot, ev, dev});
  return GM_OK;
}

struct TailCtx {
  int group, W, c;
  char *slot;
};

// Horner over the window sums in the slot; the result goes after them.
static void CUDART_CB tail_compute(void *p) {
  auto *t = static_cast<TailCtx *>(p);
  if (t->group == 1) {
    uint64_t *out = reinterpret_cast<uint64_t *>(t->slot + (size_t)t->W * sizeof(gm_host::HXyzz<gm_host::F1>));
    gm_host::horner_to_proj<gm_host::F1>(out, reinterpret_cast<const gm_host::HXyzz<gm_host::F1> *>(t->slot), t->W,
                                         t->c);
  } else {
    uint64_t *out = reinterpret_cast<uint64_t *>(t->slot + (size_t)t->W * sizeof(gm_host::HXyzz<gm_host::F2>));
    gm_host::horner_to_proj<gm_host::F2>(out, reinterpret_cast<const gm_host::HXyzz<gm_host::F2> *>(t->slot), t->W,
                                         t->c);
  }
  delete t;
}

int enqueue_host_tail(cudaStream_t s, int group, const void *d_sums, int W, int c, uint64_t *d_out) {
  const size_t elem = group == 1 ? sizeof(gm_host::HXyzz<gm_host::F1>) : sizeof(gm_host::HXyzz<gm_host::F2>);
  const size_t out_bytes = 3 * (group == 1 ? 7 : 14) * sizeof(uint64_t);
  if ((size_t)W * elem + out_bytes > TAIL_SLOT_BYTES) {
    set_last_error("too many windows for the host tail slot");
    return GM_ERR_ARG;
  }
  void *slot = nullptr;
  int rc = pinned_acquire(&slot);
  if (rc) return rc;
  auto *t = new TailCtx{group, W, c, static_cast<char *>(slot)};
  cudaError_t e = cudaMemcpyAsync(slot, d_sums, (size_t)W * elem, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) {
    pinned_release(slot);
    delete t;
    return record_error(e, "tail D2H");
  }
  e = cudaLaunchHostFunc(s, tail_compute, t);
  if (e != cudaSuccess) {
    delete t;
    // the D2H may still write the slot: release it in stream order
    enqueue_pinned_release(s, slot);
    return record_error(e, "tail host function");
  }
  e = cudaMemcpyAsync(d_out, static_cast<char *>(slot) + (size_t)W * elem, out_bytes, cudaMemcpyHostToDevice, s);
  rc = enqueue_pinned_release(s, slot);
  if (e != cudaSuccess) return record_error(e, "tail H2D");
  return rc;
}

int device_sm_count(int dev, int *sms) {
  DeviceState *st;
  int rc = device_state(dev, &st);
  if (rc) return rc;
  *sms = st->sms;
  return GM_OK;
}

int select_device(uint32_t gpu_index) {
  int count = 0;
  GM_CHECK(cudaGetDeviceCount(&count));
  if ((int)gpu_index >= count) {
    set_last_error("gpu_index out of range");
    return GM_ERR_ARG;
  }
  GM_CHECK(cudaSetDevice((int)gpu_index));
  return GM_OK;
}

int pool_alloc(int dev, cudaStream_t s, size_t bytes, void **ptr) {
  DeviceState *st;
  int rc = device_state(dev, &st);
  if (rc) return rc;
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, st->pool, s);
  if (e != cudaSuccess) {
    record_error(e, "cudaMallocFromPoolAsync");
    return GM_ERR_ALLOC;
  }
  return GM_OK;
}

// ---------------------------------------------------------------------------
// window selection (cost model in multiplication units)
//   accumulation: 10 mults per (point, non-zero window)     (madd 8M+2S)
//   reduction:    ~2.7 full adds of 14 mults per bucket      (running sums)
//   combine:      c doublings (9 mults) per window, on one thread: weighted
//                 by the serial latency against a wave of the whole GPU.
// ---------------------------------------------------------------------------
static int windows_for(int c, int limbs) { return (64 * limbs) / c + 1; }

int default_window(int group, int64_t n, int limbs) {
  (void)group;
  if (n <= 0) return 4;
  const int bits = std::min(64 * limbs, 300);
  double best = 1e300;
  int best_c = 4;
  for (int c = 3; c <= 18; c++) {
    const int W = windows_for(c, limbs);
    const int Weff = (bits + c) / c;
    const double acc = 10.0 * (double)n * Weff;
    const double red = 38.0 * (double)W * std::ldexp(1.0, c - 1);
    const double tail = 9.0 * c * Weff * 2000.0;
    // Hot buckets: a top window of few bits puts all n of its entries into a
    // handful of buckets, and a full top window (c bits, so digits above
    // 2^(c-1)) carries into one more window whose single bucket gets about
    // n/2 entries; both mean long fix-up runs and contended sort counters
    // (G1 2^17: c = 11, 2 top bits, 0.32 ms more fix-up and sort than c = 12;
    // G2 2^16: c = 11 0.63 ms, c = 13 (full top window) 0.31 ms more).
    // Scalars below r have 299 significant bits.
    const int sbits = std::min(64 * limbs, 299);
    const int top_bits = sbits - c * ((sbits + c - 1) / c - 1);
    const double hot = (top_bits <= 3 || top_bits >= c) ? 40.0 * (double)n : top_bits <= 6 ? 20.0 * (double)n : 0.0;
    const double cost = acc + red + tail + hot;
    if (cost < best) {
      best = cost;
      best_c = c;
    }
  }
  return best_c;
}

}  // namespace gm
