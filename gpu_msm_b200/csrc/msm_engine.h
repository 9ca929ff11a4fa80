// Internal interface between the C-ABI layer (capi.cu, field_kernels.cu) and
// the MSM engine (msm.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace gm {

enum {
  GM_OK = 0,
  GM_ERR_ARG = -1,
  GM_ERR_STREAM = -2,
  GM_ERR_ALLOC = -3,
  GM_ERR_CUDA = -4,
  GM_ERR_CHECK = -5,
};

int record_error(cudaError_t e, const char *where);
const char *last_error();
int select_device(uint32_t gpu_index);
int device_sm_count(int dev, int *sms);
void set_last_error(const char *msg);

// phase profiling: when enabled, msm_launch records a CUDA event on the
// launching stream at every phase boundary; profile_collect synchronises
// them and returns per-phase milliseconds.
void profile_enable(bool on);
bool profile_enabled();
void profile_mark(cudaStream_t s, const char *name);
void profile_end_call();
int profile_collect(char *names, int names_len, float *ms, int max);
// Serial window combination of one MSM on the host: copies the W window
// sums (device XYZZ) to a pinned slot, runs Horner in a stream-ordered host
// function and copies the projective result to d_out.  Not used while the
// stream is being captured.
int enqueue_host_tail(cudaStream_t s, int group, const void *d_sums, int W, int c, uint64_t *d_out);
bool host_tail_enabled();
// Pinned host slots of PINNED_SLOT_BYTES, recycled; enqueue_pinned_release
// hands a slot back once the stream reaches that point.
constexpr size_t PINNED_SLOT_BYTES = 128 * 1024;
int pinned_acquire(void **p);
void pinned_release(void *p);
int enqueue_pinned_release(cudaStream_t s, void *slot);
void set_host_tail_enabled(bool on);
// kernel launches issued by this host thread since the last reset
void count_launches(int k);
int64_t launches_and_reset();
int pool_alloc(int dev, cudaStream_t s, size_t bytes, void **ptr);
int default_window(int group, int64_t n, int limbs);

// Window sums handed to a synchronous caller in place of the stream-ordered
// host tail: the MSM copies its W window sums (XYZZ, device layout) to
// `host` (pinned, `cap` bytes), sets W and c and writes no result; the caller
// combines them (gm_host::horner_to_proj) after synchronising the stream.
struct TailHandoff {
  void *host = nullptr;
  size_t cap = 0;
  int W = 0, c = 0;
};

// Full MSM pipeline on `s`.  Either `bases` (packed records) or `ref_points`
// (reference-layout affine points; converted to Montgomery when to_mont) is
// given.  Writes the projective result (reference layout) to out_proj.  When
// err_out is non-null it receives the device consistency flag (0 = ok).
// bases_ready (optional): an event the stream waits for after the sort,
// before the bases are first read (the sort reads only the scalars).
// handoff (optional, not while capturing): the window sums go to the caller
// instead of a result in out_proj.
template <class F>
int msm_launch(cudaStream_t s, int dev, const uint4 *bases, const uint64_t *ref_points, int to_mont,
               const uint64_t *scalars, int limbs, int64_t n, uint64_t *out_proj, int c_override, uint32_t *err_out,
               cudaEvent_t bases_ready = nullptr, TailHandoff *handoff = nullptr);

}  // namespace gm
