// C-ABI entry points of include/gpu_msm_b200.h (point helpers, MSM wrappers,
// resident conversions, fixed-base batch).  The field-array entry points live
// in field_kernels.cu.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "../../include/gpu_msm_b200.h"
#include "host_arith.h"
#include "msm_engine.h"
#include "msm_kernels.cuh"

namespace {

namespace H = gm_host;

// ---------------------------------------------------------------------------
// host-side point helpers (c_wrapper.cu:12-59, 261-288 of the reference)
// ---------------------------------------------------------------------------
template <class Prj>
void proj_zero(Prj *p) {
  memset(p, 0, sizeof(*p));
}

// Fp2 helpers over the C structs
void f2_add(Fp2 &c, const Fp2 &a, const Fp2 &b) {
  H::add(c.c0.limb, a.c0.limb, b.c0.limb);
  H::add(c.c1.limb, a.c1.limb, b.c1.limb);
}
void f2_sub(Fp2 &c, const Fp2 &a, const Fp2 &b) {
  H::sub(c.c0.limb, a.c0.limb, b.c0.limb);
  H::sub(c.c1.limb, a.c1.limb, b.c1.limb);
}

// affine doubling over host arithmetic; used to build the 2^j * G tables
void g1_affine_double(G1Point &r, const G1Point &p) {
  if (p.infinity || H::is_zero(p.y.limb)) {
    memset(&r, 0, sizeof(r));
    r.infinity = true;
    return;
  }
  uint64_t xx[7], m[7], ty[7], ti[7], lam[7], l2[7], tx[7], x3[7], d[7], y3[7];
  H::mont_mul(xx, p.x.limb, p.x.limb);
  H::add(m, xx, xx);
  H::add(m, m, xx);
  H::add(ty, p.y.limb, p.y.limb);
  H::mont_inv(ti, ty);
  H::mont_mul(lam, m, ti);
  H::mont_mul(l2, lam, lam);
  H::add(tx, p.x.limb, p.x.limb);
  H::sub(x3, l2, tx);
  H::sub(d, p.x.limb, x3);
  H::mont_mul(y3, lam, d);
  H::sub(y3, y3, p.y.limb);
  G1Point out;
  memset(&out, 0, sizeof(out));
  memcpy(out.x.limb, x3, sizeof(x3));
  memcpy(out.y.limb, y3, sizeof(y3));
  r = out;
}

void g2_affine_double(G2Point &r, const G2Point &p) {
  if (p.infinity || H::fp2_is_zero(p.y)) {
    memset(&r, 0, sizeof(r));
    r.infinity = true;
    return;
  }
  Fp2 xx, m, ty, ti, lam, l2, tx, x3, d, y3;
  H::fp2_mul(xx, p.x, p.x);
  f2_add(m, xx, xx);
  f2_add(m, m, xx);
  f2_add(ty, p.y, p.y);
  H::fp2_inv(ti, ty);
  H::fp2_mul(lam, m, ti);
  H::fp2_mul(l2, lam, lam);
  f2_add(tx, p.x, p.x);
  f2_sub(x3, l2, tx);
  f2_sub(d, p.x, x3);
  H::fp2_mul(y3, lam, d);
  f2_sub(y3, y3, p.y);
  G2Point out;
  memset(&out, 0, sizeof(out));
  out.x = x3;
  out.y = y3;
  r = out;
}

// Generators in standard form (src/curve.cu:786-814)
const uint64_t G1X[7] = {0x3bf9166c8236f4faULL, 0x8bc02b7cbe6a9e8dULL, 0x11c1e56b3e4bc80bULL, 0x6b20d782901a6f62ULL,
                         0x2ce8c34265bf3841ULL, 0x11b73d3d76ae9851ULL, 0x326ed6bd777fc6a3ULL};
const uint64_t G1Y[7] = {0xfe6f792612016b30ULL, 0x22db0ce6034a9db9ULL, 0xb9093f32002756daULL, 0x39d7f424b6660204ULL,
                         0xf843c947aa57f571ULL, 0xd6d62d244e413636ULL, 0x1a7caf4a4d3887a6ULL};
const uint64_t G2X0[7] = {0x0e529ee4dce9991dULL, 0xd6ebaf149094f1ccULL, 0x043c6bf16312d638ULL, 0x062b61439640e885ULL,
                          0x18dad8ed784dd225ULL, 0xa57c0038441f7d15ULL, 0x21f8d4a76f74541aULL};
const uint64_t G2X1[7] = {0xcaf5185423a7d23aULL, 0x7cef6acb145b6413ULL, 0x2879dd439b019b8bULL, 0x71449cdeca4f0007ULL,
                          0xdebaf4a2c5534527ULL, 0xa1b4e791d1b86560ULL, 0x1e0f563c601bb8dcULL};
const uint64_t G2Y0[7] = {0x274315837455b919ULL, 0x82039e4221ff3507ULL, 0x00346cebad16a036ULL, 0x0177bfd6654e681eULL,
                          0xddff621b5db3f897ULL, 0x0cc61570301497a7ULL, 0x115ea2305a78f646ULL};
const uint64_t G2Y1[7] = {0x392236e9cf2976c2ULL, 0xd8ab17c84b9f03cdULL, 0x8a8e6755f9d82fd1ULL, 0x7532834528cd5a64ULL,
                          0x0b0bcc3fb6f2161cULL, 0x76a2ffcb7d47679dULL, 0x25ed2192b203c1feULL};

constexpr int MAX_TABLE_BITS = 64 * gm::MAX_SCALAR_LIMBS;

// Packed records of 2^j * G, j < 512, Montgomery form.
std::vector<uint32_t> generator_table(int group) {
  const int u32_per_rec = (group == 1 ? gm::Rec<gm::Fp>::U4 : gm::Rec<gm::Fp2>::U4) * 4;
  std::vector<uint32_t> tab((size_t)MAX_TABLE_BITS * u32_per_rec, 0);
  auto put = [&](int j, const uint64_t *words, int nwords, int inf) {
    uint32_t *r = &tab[(size_t)j * u32_per_rec];
    for (int k = 0; k < nwords; k++) {
      r[2 * k] = (uint32_t)words[k];
      r[2 * k + 1] = (uint32_t)(words[k] >> 32);
    }
    r[2 * nwords] = inf;
  };
  if (group == 1) {
    G1Point g;
    memset(&g, 0, sizeof(g));
    H::to_mont(g.x.limb, G1X);
    H::to_mont(g.y.limb, G1Y);
    for (int j = 0; j < MAX_TABLE_BITS; j++) {
      uint64_t w[14];
      memcpy(w, g.x.limb, 56);
      memcpy(w + 7, g.y.limb, 56);
      put(j, w, 14, g.infinity ? 1 : 0);
      g1_affine_double(g, g);
    }
  } else {
    G2Point g;
    memset(&g, 0, sizeof(g));
    H::to_mont(g.x.c0.limb, G2X0);
    H::to_mont(g.x.c1.limb, G2X1);
    H::to_mont(g.y.c0.limb, G2Y0);
    H::to_mont(g.y.c1.limb, G2Y1);
    for (int j = 0; j < MAX_TABLE_BITS; j++) {
      uint64_t w[28];
      memcpy(w, &g.x, 112);
      memcpy(w + 14, &g.y, 112);
      put(j, w, 28, g.infinity ? 1 : 0);
      g2_affine_double(g, g);
    }
  }
  return tab;
}

std::mutex g_tab_mu;
std::map<std::pair<int, int>, void *> g_tab;  // (device, group) -> device table

int device_generator_table(int dev, int group, const uint4 **out) {
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto key = std::make_pair(dev, group);
  auto it = g_tab.find(key);
  if (it == g_tab.end()) {
    std::vector<uint32_t> tab = generator_table(group);
    void *d = nullptr;
    cudaError_t e = cudaMalloc(&d, tab.size() * sizeof(uint32_t));
    if (e != cudaSuccess) return gm::record_error(e, "cudaMalloc(generator table)");
    e = cudaMemcpy(d, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return gm::record_error(e, "cudaMemcpy(generator table)");
    it = g_tab.emplace(key, d).first;
  }
  *out = (const uint4 *)it->second;
  return gm::GM_OK;
}

// out[i] = k_i * G as canonical Montgomery affine (reference layout)
template <class F>
__global__ void k_generator_mul(uint64_t *__restrict__ out, const uint4 *__restrict__ table,
                                const uint64_t *__restrict__ scalars, int limbs, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  using T = typename F::T;
  gm::xyzz_t<F> acc;
  gm::xyzz_set_inf(acc);
  for (int l = 0; l < limbs; l++) {
    uint64_t k = scalars[i * limbs + l];
    while (k) {
      const int b = __ffsll((long long)k) - 1;
      k &= k - 1;
      T x, y;
      gm::load_base<F>(x, y, table + (size_t)(64 * l + b) * gm::Rec<F>::U4);
      gm::xyzz_madd<F>(acc, x, y);
    }
  }
  constexpr int Hw = F::LIMBS / 2;
  uint64_t *dst = out + i * (2 * Hw + 1);
  if (gm::xyzz_is_inf(acc)) {
    for (int k = 0; k < 2 * Hw; k++) dst[k] = 0;
    dst[2 * Hw] = 1;  // infinity flag byte, pad bytes zero
    return;
  }
  const T I = F::inv(F::mul(acc.ZZ, acc.ZZZ));
  T x = F::mul(acc.X, F::mul(I, acc.ZZZ));
  T y = F::mul(acc.Y, F::mul(I, acc.ZZ));
  gm::store_ref<F>(dst, x);
  gm::store_ref<F>(dst + Hw, y);
  dst[2 * Hw] = 0;
}

// in-place standard -> Montgomery of reference-layout points (curve.cu:2343)
template <class F>
__global__ void k_to_mont_ref(uint64_t *__restrict__ pts, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  constexpr int Hw = F::LIMBS / 2;
  uint64_t *p = pts + i * (2 * Hw + 1);
  if (reinterpret_cast<const uint8_t *>(p + 2 * Hw)[0]) return;
  typename F::T x, y;
  gm::load_ref<F>(x, p);
  gm::load_ref<F>(y, p + Hw);
  x = gm::field_to_mont<F>(x);
  y = gm::field_to_mont<F>(y);
  gm::store_ref<F>(p, x);
  gm::store_ref<F>(p + Hw, y);
}

// out = sum of n projective points (reference layout); one thread.  Combines
// the partial results of an MSM sharded across devices or batches.
template <class F>
__global__ void k_proj_sum(uint64_t *__restrict__ out, const uint64_t *__restrict__ in, int n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  constexpr int Hw = F::LIMBS / 2;
  gm::xyzz_t<F> acc;
  gm::xyzz_set_inf(acc);
  for (int i = 0; i < n; i++) {
    typename F::T X, Y, Z;
    gm::load_ref<F>(X, in + (size_t)i * 3 * Hw);
    gm::load_ref<F>(Y, in + (size_t)i * 3 * Hw + Hw);
    gm::load_ref<F>(Z, in + (size_t)i * 3 * Hw + 2 * Hw);
    gm::xyzz_t<F> p;
    gm::proj_to_xyzz<F>(p, X, Y, Z);
    gm::xyzz_add_cold<F>(acc, p);
  }
  typename F::T X, Y, Z;
  gm::xyzz_to_proj<F>(X, Y, Z, acc);
  gm::store_ref<F>(out, X);
  gm::store_ref<F>(out + Hw, Y);
  gm::store_ref<F>(out + 2 * Hw, Z);
}

// host arithmetic of a device field: gm::Fp -> gm_host::F1, gm::Fp2 -> F2
template <class F>
using HostField = typename std::conditional<sizeof(typename F::T) == sizeof(gm::fp_t), gm_host::F1, gm_host::F2>::type;

template <class F, class Aff, class Prj>
int host_msm(Prj *result, const Aff *points, const uint64_t *scalars, int limbs, int n, uint32_t gpu_index,
             int to_mont) {
  if (result == nullptr || n < 0 || (n > 0 && (points == nullptr || scalars == nullptr))) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  if (n == 0) {
    proj_zero(result);
    return gm::GM_OK;
  }
  // the scalars go first on s; the points follow on a second stream, so
  // their copy overlaps the sort (which reads only the scalars)
  cudaStream_t s, s2;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return gm::GM_ERR_STREAM;
  if (cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(s);
    return gm::GM_ERR_STREAM;
  }
  cudaEvent_t alloc_done, pts_done;
  if (cudaEventCreateWithFlags(&alloc_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaStreamDestroy(s);
    cudaStreamDestroy(s2);
    return gm::GM_ERR_STREAM;
  }
  if (cudaEventCreateWithFlags(&pts_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaEventDestroy(alloc_done);
    cudaStreamDestroy(s);
    cudaStreamDestroy(s2);
    return gm::GM_ERR_STREAM;
  }
  const size_t pts_bytes = (size_t)n * sizeof(Aff), sc_bytes = (size_t)n * limbs * sizeof(uint64_t);
  const size_t o_sc = (pts_bytes + 255) / 256 * 256;
  const size_t o_res = o_sc + (sc_bytes + 255) / 256 * 256;
  const size_t o_err = o_res + 512;
  char *buf = nullptr;
  // the window sums come back to this thread, which runs the Horner tail
  // itself: no stream host function and no result copy in and out
  void *slot = nullptr;
  uint32_t *err_host = nullptr;
  gm::TailHandoff handoff;
  cudaError_t e = cudaSuccess;
  rc = gm::pinned_acquire(&slot);
  if (rc == gm::GM_OK) {
    err_host = static_cast<uint32_t *>(slot);
    *err_host = 0;
    handoff.host = static_cast<char *>(slot) + 256;
    handoff.cap = gm::PINNED_SLOT_BYTES - 256;
    rc = gm::pool_alloc((int)gpu_index, s, o_err + 256, (void **)&buf);
  }
  if (rc == gm::GM_OK) {
    e = cudaMemcpyAsync(buf + o_sc, scalars, sc_bytes, cudaMemcpyHostToDevice, s);
    // the points' stream may use the buffer once its allocation is ordered
    if (e == cudaSuccess) e = cudaEventRecord(alloc_done, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, alloc_done, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf, points, pts_bytes, cudaMemcpyHostToDevice, s2);
    if (e == cudaSuccess) e = cudaEventRecord(pts_done, s2);
    if (e == cudaSuccess) {
      rc = gm::msm_launch<F>(s, (int)gpu_index, nullptr, (const uint64_t *)buf, to_mont,
                             (const uint64_t *)(buf + o_sc), limbs, n, (uint64_t *)(buf + o_res), 0,
                             (uint32_t *)(buf + o_err), pts_done, &handoff);
      if (rc == gm::GM_OK) e = cudaMemcpyAsync(err_host, buf + o_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    }
    // s waited for pts_done inside msm_launch, or waits here on an early error
    cudaStreamWaitEvent(s, pts_done, 0);
    cudaFreeAsync(buf, s);
  }
  cudaError_t se = cudaStreamSynchronize(s);
  cudaError_t se2 = cudaStreamSynchronize(s2);
  cudaEventDestroy(alloc_done);
  cudaEventDestroy(pts_done);
  cudaStreamDestroy(s);
  cudaStreamDestroy(s2);
  const uint32_t flag = err_host ? *err_host : 0u;
  if (rc == gm::GM_OK && e == cudaSuccess && se == cudaSuccess && se2 == cudaSuccess && flag == 0)
    gm_host::horner_to_proj<HostField<F>>(reinterpret_cast<uint64_t *>(result),
                                          reinterpret_cast<const gm_host::HXyzz<HostField<F>> *>(handoff.host),
                                          handoff.W, handoff.c);
  if (slot) gm::pinned_release(slot);
  if (rc) return rc;
  if (e != cudaSuccess) return gm::record_error(e, "host_msm copy");
  if (se != cudaSuccess) return gm::record_error(se, "host_msm sync");
  if (se2 != cudaSuccess) return gm::record_error(se2, "host_msm sync");
  if (flag) return gm::GM_ERR_CHECK;
  return gm::GM_OK;
}

// One non-blocking helper stream per device for the points' copy of the
// asynchronous host-buffer MSM (created on first use, kept for the process).
std::mutex g_copy_mu;
std::map<int, cudaStream_t> g_copy_streams;

int copy_stream(int dev, cudaStream_t *out) {
  std::lock_guard<std::mutex> lk(g_copy_mu);
  auto it = g_copy_streams.find(dev);
  if (it == g_copy_streams.end()) {
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return gm::GM_ERR_STREAM;
    it = g_copy_streams.emplace(dev, cs).first;
  }
  *out = it->second;
  return gm::GM_OK;
}

// Host-buffer MSM enqueued on the caller's stream s: scalars copied on s,
// points on the helper stream (so that their copy overlaps the sort), the
// MSM, then the result (and the consistency flag) copied back to host
// memory; nothing waits on the host.  Per-call events are released once
// the stream has passed them.
template <class F, class Aff, class Prj>
int host_msm_async(cudaStream_t s, uint32_t gpu_index, Prj *result, const Aff *points, const uint64_t *scalars,
                   int limbs, int n, int to_mont, uint32_t *err_flag) {
  if (result == nullptr || n < 0 || (n > 0 && (points == nullptr || scalars == nullptr))) return gm::GM_ERR_ARG;
  if (limbs < 1 || limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  const size_t pts_bytes = (size_t)n * sizeof(Aff), sc_bytes = (size_t)n * limbs * sizeof(uint64_t);
  const size_t o_sc = (pts_bytes + 255) / 256 * 256;
  const size_t o_res = o_sc + (sc_bytes + 255) / 256 * 256;
  const size_t o_err = o_res + 512;
  char *buf = nullptr;
  rc = gm::pool_alloc((int)gpu_index, s, o_err + 256, (void **)&buf);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
  if (n == 0) {  // the identity: Z = 0 (reference layout, all words zero)
    e = cudaMemsetAsync(buf + o_res, 0, sizeof(Prj), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(result, buf + o_res, sizeof(Prj), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && err_flag) e = cudaMemsetAsync(buf + o_err, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess && err_flag)
      e = cudaMemcpyAsync(err_flag, buf + o_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(buf, s);
    return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "host_msm_async");
  }
  cudaStream_t s2;
  rc = copy_stream((int)gpu_index, &s2);
  if (rc) {
    cudaFreeAsync(buf, s);
    return rc;
  }
  cudaEvent_t alloc_done, pts_done;
  if (cudaEventCreateWithFlags(&alloc_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaFreeAsync(buf, s);
    return gm::GM_ERR_STREAM;
  }
  if (cudaEventCreateWithFlags(&pts_done, cudaEventDisableTiming) != cudaSuccess) {
    cudaEventDestroy(alloc_done);
    cudaFreeAsync(buf, s);
    return gm::GM_ERR_STREAM;
  }
  e = cudaMemcpyAsync(buf + o_sc, scalars, sc_bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(alloc_done, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, alloc_done, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf, points, pts_bytes, cudaMemcpyHostToDevice, s2);
  if (e == cudaSuccess) e = cudaEventRecord(pts_done, s2);
  if (e == cudaSuccess) {
    rc = gm::msm_launch<F>(s, (int)gpu_index, nullptr, (const uint64_t *)buf, to_mont, (const uint64_t *)(buf + o_sc),
                           limbs, n, (uint64_t *)(buf + o_res), 0, (uint32_t *)(buf + o_err), pts_done);
    if (rc == gm::GM_OK) {
      e = cudaMemcpyAsync(result, buf + o_res, sizeof(Prj), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && err_flag)
        e = cudaMemcpyAsync(err_flag, buf + o_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    }
  }
  // s waited for pts_done inside msm_launch, or waits here on an early error
  cudaStreamWaitEvent(s, pts_done, 0);
  cudaFreeAsync(buf, s);
  cudaEventDestroy(alloc_done);
  cudaEventDestroy(pts_done);
  if (rc) return rc;
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "host_msm_async");
}

}  // namespace

extern "C" {

// ---- Part 1: reference C-ABI ------------------------------------------------

void affine_to_projective_g1_wrapper(G1ProjectivePoint *proj, const G1Point *affine) {
  if (affine->infinity) {
    proj_zero(proj);
    return;
  }
  G1ProjectivePoint r;
  r.X = affine->x;
  r.Y = affine->y;
  H::one_mont(r.Z.limb);
  *proj = r;
}

void affine_to_projective_g2_wrapper(G2ProjectivePoint *proj, const G2Point *affine) {
  if (affine->infinity) {
    proj_zero(proj);
    return;
  }
  G2ProjectivePoint r;
  r.X = affine->x;
  r.Y = affine->y;
  H::one_mont(r.Z.c0.limb);
  memset(&r.Z.c1, 0, sizeof(r.Z.c1));
  *proj = r;
}

void projective_to_affine_g1_wrapper(G1Point *affine, const G1ProjectivePoint *proj) {
  G1Point r;
  memset(&r, 0, sizeof(r));
  if (H::is_zero(proj->Z.limb)) {
    r.infinity = true;
  } else {
    uint64_t zi[7];
    H::mont_inv(zi, proj->Z.limb);
    H::mont_mul(r.x.limb, proj->X.limb, zi);
    H::mont_mul(r.y.limb, proj->Y.limb, zi);
  }
  *affine = r;
}

void projective_to_affine_g2_wrapper(G2Point *affine, const G2ProjectivePoint *proj) {
  G2Point r;
  memset(&r, 0, sizeof(r));
  if (H::fp2_is_zero(proj->Z)) {
    r.infinity = true;
  } else {
    Fp2 zi;
    H::fp2_inv(zi, proj->Z);
    H::fp2_mul(r.x, proj->X, zi);
    H::fp2_mul(r.y, proj->Y, zi);
  }
  *affine = r;
}

void g1_point_at_infinity_wrapper(G1Point *point) {
  memset(point, 0, sizeof(*point));
  point->infinity = true;
}
void g2_point_at_infinity_wrapper(G2Point *point) {
  memset(point, 0, sizeof(*point));
  point->infinity = true;
}
void g1_projective_point_at_infinity_wrapper(G1ProjectivePoint *point) { proj_zero(point); }
void g2_projective_point_at_infinity_wrapper(G2ProjectivePoint *point) { proj_zero(point); }
bool g1_is_infinity_wrapper(const G1Point *point) { return point->infinity; }
bool g2_is_infinity_wrapper(const G2Point *point) { return point->infinity; }

int g1_msm_wrapper(G1ProjectivePoint *result, const G1Point *points, const uint64_t *scalars, int n,
                   uint32_t gpu_index) {
  if (n <= 0) return gm::GM_ERR_ARG;  // c_wrapper.cu:71-73
  return host_msm<gm::Fp>(result, points, scalars, 1, n, gpu_index, /*to_mont=*/1);
}

int g2_msm_wrapper(G2ProjectivePoint *result, const G2Point *points, const uint64_t *scalars, int n,
                   uint32_t gpu_index) {
  if (n <= 0) return gm::GM_ERR_ARG;  // c_wrapper.cu:182-184
  return host_msm<gm::Fp2>(result, points, scalars, 1, n, gpu_index, /*to_mont=*/0);
}

void g1_from_montgomery_wrapper(G1Point *result, const G1Point *point) {
  G1Point r;
  memset(&r, 0, sizeof(r));
  if (point->infinity) {
    r.infinity = true;
  } else {
    H::from_mont(r.x.limb, point->x.limb);
    H::from_mont(r.y.limb, point->y.limb);
  }
  *result = r;
}

void g2_from_montgomery_wrapper(G2Point *result, const G2Point *point) {
  G2Point r;
  memset(&r, 0, sizeof(r));
  if (point->infinity) {
    r.infinity = true;
  } else {
    H::from_mont(r.x.c0.limb, point->x.c0.limb);
    H::from_mont(r.x.c1.limb, point->x.c1.limb);
    H::from_mont(r.y.c0.limb, point->y.c0.limb);
    H::from_mont(r.y.c1.limb, point->y.c1.limb);
  }
  *result = r;
}

void fp_to_montgomery_wrapper(Fp *result, const Fp *value) {
  uint64_t t[7];
  H::to_mont(t, value->limb);
  memcpy(result->limb, t, sizeof(t));
}

void init_device_generators(gm_stream_t stream, uint32_t gpu_index) {
  (void)stream;
  gm::select_device(gpu_index);
}

// ---- Part 2 -----------------------------------------------------------------

int g1_msm_limbs_wrapper(G1ProjectivePoint *result, const G1Point *points, const uint64_t *scalars, int scalar_limbs,
                         int n, uint32_t gpu_index, int points_montgomery) {
  if (scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  return host_msm<gm::Fp>(result, points, scalars, scalar_limbs, n, gpu_index, points_montgomery ? 0 : 1);
}

int g2_msm_limbs_wrapper(G2ProjectivePoint *result, const G2Point *points, const uint64_t *scalars, int scalar_limbs,
                         int n, uint32_t gpu_index, int points_montgomery) {
  if (scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  return host_msm<gm::Fp2>(result, points, scalars, scalar_limbs, n, gpu_index, points_montgomery ? 0 : 1);
}

int gm_g1_msm_host_async(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *result, const G1Point *points,
                         const uint64_t *scalars, int scalar_limbs, int n, int points_montgomery, uint32_t *err_flag) {
  return host_msm_async<gm::Fp>((cudaStream_t)stream, gpu_index, result, points, scalars, scalar_limbs, n,
                                points_montgomery ? 0 : 1, err_flag);
}

int gm_g2_msm_host_async(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *result, const G2Point *points,
                         const uint64_t *scalars, int scalar_limbs, int n, int points_montgomery, uint32_t *err_flag) {
  return host_msm_async<gm::Fp2>((cudaStream_t)stream, gpu_index, result, points, scalars, scalar_limbs, n,
                                 points_montgomery ? 0 : 1, err_flag);
}

int gm_g1_msm_device_c(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                       const uint64_t *d_scalars, int scalar_limbs, int n, int window_bits) {
  if (d_result == nullptr || n < 0 || (n > 0 && (d_points == nullptr || d_scalars == nullptr))) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  return gm::msm_launch<gm::Fp>((cudaStream_t)stream, (int)gpu_index, nullptr, (const uint64_t *)d_points, 0, d_scalars,
                                scalar_limbs, n, (uint64_t *)d_result, window_bits, nullptr);
}

int gm_g2_msm_device_c(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                       const uint64_t *d_scalars, int scalar_limbs, int n, int window_bits) {
  if (d_result == nullptr || n < 0 || (n > 0 && (d_points == nullptr || d_scalars == nullptr))) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  return gm::msm_launch<gm::Fp2>((cudaStream_t)stream, (int)gpu_index, nullptr, (const uint64_t *)d_points, 0, d_scalars,
                                 scalar_limbs, n, (uint64_t *)d_result, window_bits, nullptr);
}

}  // extern "C"

namespace {

// Projective sum -> affine result on the host, ordered on the stream: the
// pinned slot holds the projective input at offset 0 and the affine output
// at AFF_OFF.
constexpr size_t AFF_OFF = 512;

void CUDART_CB g1_to_affine_cb(void *slot) {
  auto *base = static_cast<char *>(slot);
  projective_to_affine_g1_wrapper(reinterpret_cast<G1Point *>(base + AFF_OFF),
                                  reinterpret_cast<const G1ProjectivePoint *>(base));
}
void CUDART_CB g2_to_affine_cb(void *slot) {
  auto *base = static_cast<char *>(slot);
  projective_to_affine_g2_wrapper(reinterpret_cast<G2Point *>(base + AFF_OFF),
                                  reinterpret_cast<const G2ProjectivePoint *>(base));
}

template <class F, class Aff, class Prj>
int msm_affine(gm_stream_t stream, uint32_t gpu_index, Aff *d_result, const Aff *d_points, const uint64_t *d_scalars,
               int scalar_limbs, int n, cudaHostFn_t to_affine) {
  if (d_result == nullptr || n < 0 || (n > 0 && (d_points == nullptr || d_scalars == nullptr))) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    Aff inf;
    memset(&inf, 0, sizeof(inf));
    inf.infinity = true;
    void *slot = nullptr;
    rc = gm::pinned_acquire(&slot);
    if (rc) return rc;
    memcpy(slot, &inf, sizeof(inf));
    cudaError_t e = cudaMemcpyAsync(d_result, slot, sizeof(Aff), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return gm::record_error(e, "msm_affine copy");
    return gm::enqueue_pinned_release(s, slot);
  }
  void *tmp = nullptr;
  rc = gm::pool_alloc((int)gpu_index, s, sizeof(Prj), &tmp);
  if (rc) return rc;
  rc = gm::msm_launch<F>(s, (int)gpu_index, nullptr, (const uint64_t *)d_points, 0, d_scalars, scalar_limbs, n,
                         (uint64_t *)tmp, 0, nullptr);
  if (rc) return rc;
  void *slot = nullptr;
  rc = gm::pinned_acquire(&slot);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(slot, tmp, sizeof(Prj), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(s, to_affine, slot);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_result, static_cast<char *>(slot) + AFF_OFF, sizeof(Aff), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return gm::record_error(e, "msm_affine");
  rc = gm::enqueue_pinned_release(s, slot);
  if (rc) return rc;
  e = cudaFreeAsync(tmp, s);
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "msm_affine free");
}

}  // namespace

extern "C" {

int gm_g1_msm_device_affine(gm_stream_t stream, uint32_t gpu_index, G1Point *d_result, const G1Point *d_points,
                            const uint64_t *d_scalars, int scalar_limbs, int n) {
  return msm_affine<gm::Fp, G1Point, G1ProjectivePoint>(stream, gpu_index, d_result, d_points, d_scalars, scalar_limbs,
                                                        n, g1_to_affine_cb);
}

int gm_g2_msm_device_affine(gm_stream_t stream, uint32_t gpu_index, G2Point *d_result, const G2Point *d_points,
                            const uint64_t *d_scalars, int scalar_limbs, int n) {
  return msm_affine<gm::Fp2, G2Point, G2ProjectivePoint>(stream, gpu_index, d_result, d_points, d_scalars,
                                                         scalar_limbs, n, g2_to_affine_cb);
}

int gm_g1_msm_device(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_result, const G1Point *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, int n) {
  return gm_g1_msm_device_c(stream, gpu_index, d_result, d_points, d_scalars, scalar_limbs, n, 0);
}

int gm_g2_msm_device(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_result, const G2Point *d_points,
                     const uint64_t *d_scalars, int scalar_limbs, int n) {
  return gm_g2_msm_device_c(stream, gpu_index, d_result, d_points, d_scalars, scalar_limbs, n, 0);
}

int gm_msm_default_window(int group, int64_t n, int scalar_limbs) { return gm::default_window(group, n, scalar_limbs); }

int gm_g1_to_montgomery_batch(gm_stream_t stream, uint32_t gpu_index, G1Point *d_points, int n) {
  if (n < 0 || (n > 0 && d_points == nullptr)) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  k_to_mont_ref<gm::Fp><<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>((uint64_t *)d_points, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_to_mont_ref");
}

int gm_g2_to_montgomery_batch(gm_stream_t stream, uint32_t gpu_index, G2Point *d_points, int n) {
  if (n < 0 || (n > 0 && d_points == nullptr)) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  k_to_mont_ref<gm::Fp2><<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>((uint64_t *)d_points, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_to_mont_ref");
}

int gm_g1_generator_mul_batch(gm_stream_t stream, uint32_t gpu_index, G1Point *d_out, const uint64_t *d_scalars,
                              int scalar_limbs, int n) {
  if (n < 0 || scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  const uint4 *tab;
  rc = device_generator_table((int)gpu_index, 1, &tab);
  if (rc) return rc;
  k_generator_mul<gm::Fp><<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>((uint64_t *)d_out, tab, d_scalars,
                                                                             scalar_limbs, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_generator_mul");
}

int gm_g2_generator_mul_batch(gm_stream_t stream, uint32_t gpu_index, G2Point *d_out, const uint64_t *d_scalars,
                              int scalar_limbs, int n) {
  if (n < 0 || scalar_limbs < 1 || scalar_limbs > gm::MAX_SCALAR_LIMBS) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc || n == 0) return rc;
  const uint4 *tab;
  rc = device_generator_table((int)gpu_index, 2, &tab);
  if (rc) return rc;
  k_generator_mul<gm::Fp2><<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>((uint64_t *)d_out, tab, d_scalars,
                                                                              scalar_limbs, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_generator_mul");
}

int gm_g1_sum_projective(gm_stream_t stream, uint32_t gpu_index, G1ProjectivePoint *d_out,
                         const G1ProjectivePoint *d_in, int n) {
  if (n < 0 || d_out == nullptr || (n > 0 && d_in == nullptr)) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  k_proj_sum<gm::Fp><<<1, 1, 0, (cudaStream_t)stream>>>((uint64_t *)d_out, (const uint64_t *)d_in, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_proj_sum");
}

int gm_g2_sum_projective(gm_stream_t stream, uint32_t gpu_index, G2ProjectivePoint *d_out,
                         const G2ProjectivePoint *d_in, int n) {
  if (n < 0 || d_out == nullptr || (n > 0 && d_in == nullptr)) return gm::GM_ERR_ARG;
  int rc = gm::select_device(gpu_index);
  if (rc) return rc;
  k_proj_sum<gm::Fp2><<<1, 1, 0, (cudaStream_t)stream>>>((uint64_t *)d_out, (const uint64_t *)d_in, n);
  gm::count_launches(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? gm::GM_OK : gm::record_error(e, "k_proj_sum");
}

}  // extern "C"

// Self-test of the host arithmetic used by the window combination.
namespace {
uint64_t st_next(uint64_t &s) {
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return s;
}
void st_fp(gm_host::HFp &a, uint64_t &s) {
  for (int i = 0; i < 7; i++) a.v[i] = st_next(s);
  a.v[6] &= 0x0fffffffffffffffULL;  // < 2^444 < p
}
template <class F>
bool st_same_affine(const gm_host::HXyzz<F> &a, const uint64_t *proj) {
  // XYZZ a against projective (X, Y, Z): X_a ZZZ_a Z == X ZZ_a ZZZ_a ... compare
  // x = X_a / ZZ_a with X / Z and y = Y_a / ZZZ_a with Y / Z by cross products
  typename F::T X, Y, Z, l, r;
  memcpy(&X, proj, sizeof(X));
  memcpy(&Y, proj + F::WORDS, sizeof(Y));
  memcpy(&Z, proj + 2 * F::WORDS, sizeof(Z));
  const bool inf_a = gm_host::hx_is_inf(a), inf_b = F::is_zero(Z);
  if (inf_a || inf_b) return inf_a == inf_b;
  F::mul(l, a.X, Z);
  F::mul(r, X, a.ZZ);
  if (memcmp(&l, &r, sizeof(l))) return false;
  F::mul(l, a.Y, Z);
  F::mul(r, Y, a.ZZZ);
  return memcmp(&l, &r, sizeof(l)) == 0;
}
template <class F>
int st_horner(uint64_t &seed, void (*fill)(typename F::T &, uint64_t &)) {
  gm_host::HXyzz<F> sums[9];
  for (int w = 0; w < 9; w++) {
    fill(sums[w].X, seed);
    fill(sums[w].Y, seed);
    typename F::T z;
    fill(z, seed);
    F::sqr(sums[w].ZZ, z);
    F::mul(sums[w].ZZZ, sums[w].ZZ, z);
  }
  memset(&sums[3], 0, sizeof(sums[3]));  // an empty window
  uint64_t out[3 * 14];
  gm_host::HXyzz<F> ref;
  for (int c : {1, 5, 13}) {
    gm_host::horner_to_proj<F>(out, sums, 9, c);
    gm_host::horner_xyzz<F>(ref, sums, 9, c);
    if (!st_same_affine<F>(ref, out)) return 1;
  }
  return 0;
}
void st_f1(gm_host::HFp &a, uint64_t &s) { st_fp(a, s); }
void st_f2(gm_host::HFp2 &a, uint64_t &s) {
  st_fp(a.c0, s);
  st_fp(a.c1, s);
}
}  // namespace

extern "C" {

int gm_host_selftest(void) {
  uint64_t seed = 0x9e3779b97f4a7c15ULL;
  // squaring against the general product: edge values and random elements
  gm_host::HFp a, x, y;
  for (int k = 0; k < 2000; k++) {
    if (k < 4) {
      memset(&a, 0, sizeof(a));
      if (k == 1) a.v[0] = 1;
      if (k >= 2) {
        memcpy(a.v, gm_host::P, sizeof(a.v));
        a.v[0] -= (uint64_t)(k - 1);  // p - 1, p - 2
      }
    } else {
      st_fp(a, seed);
    }
    gm_host::F1::sqr(x, a);
    gm_host::F1::mul(y, a, a);
    if (memcmp(&x, &y, sizeof(x))) return 1;
  }
  for (int k = 0; k < 500; k++) {
    gm_host::HFp2 b, u, v;
    st_f2(b, seed);
    gm_host::F2::sqr(u, b);
    gm_host::F2::mul(v, b, b);
    if (memcmp(&u, &v, sizeof(u))) return 2;
  }
  if (st_horner<gm_host::F1>(seed, st_f1)) return 3;
  if (st_horner<gm_host::F2>(seed, st_f2)) return 4;
  return 0;
}

int gm_g1_sum_projective_host(G1ProjectivePoint *out, const G1ProjectivePoint *in, int n) {
  if (n < 0 || out == nullptr || (n > 0 && in == nullptr)) return gm::GM_ERR_ARG;
  gm_host::HXyzz<gm_host::F1> acc;
  memset(&acc, 0, sizeof(acc));
  for (int i = 0; i < n; i++) {
    // homogeneous (X, Y, Z) -> XYZZ (X Z, Y Z^2, Z^2, Z^3)
    gm_host::HXyzz<gm_host::F1> p;
    memset(&p, 0, sizeof(p));
    if (!gm_host::is_zero(in[i].Z.limb)) {
      gm_host::F1::T X, Y, Z;
      memcpy(X.v, in[i].X.limb, 56);
      memcpy(Y.v, in[i].Y.limb, 56);
      memcpy(Z.v, in[i].Z.limb, 56);
      gm_host::F1::mul(p.ZZ, Z, Z);
      gm_host::F1::mul(p.ZZZ, p.ZZ, Z);
      gm_host::F1::mul(p.X, X, Z);
      gm_host::F1::mul(p.Y, Y, p.ZZ);
    }
    gm_host::hx_add(acc, p);
  }
  uint64_t words[21];
  gm_host::horner_to_proj<gm_host::F1>(words, &acc, 1, 0);
  memcpy(out, words, sizeof(words));
  return gm::GM_OK;
}

const char *gm_last_error(void) { return gm::last_error(); }

}  // extern "C"
