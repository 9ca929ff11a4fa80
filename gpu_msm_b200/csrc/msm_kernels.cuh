// Pippenger bucket-method kernels for BLS12-446 G1/G2 on sm_100a.
//
// Pipeline for one MSM  sum_i k_i * P_i  (replaces the per-window host loop of
// pdroalves/gpu_msm src/curve.cu:2538-2677 and the affine multi-limb path
// src/curve.cu:2763-2820):
//
//  1-3. k_sort_*  signed c-bit digit decomposition of every scalar and a
//                  stable radix sort of the (point, sign) entries by bucket
//                  key  key = w*B + |d|-1  (B = 2^(c-1) buckets per window),
//                  with the bucket offsets (msm_sort.cuh; k_scan_* below are
//                  its prefix sums).
//  4. k_accumulate every thread sums an equal-length slice of the sorted
//                  entries with XYZZ mixed additions; buckets that fit in a
//                  slice are written directly, the edge pieces of buckets that
//                  straddle slices are written as partials.
//  5. k_fixup_*    the slice that opened a straddling bucket adds the
//                  partials of the following slices (msm_reduce.cuh).
//  6. k_red_*      per window, sum_b (b+1)*Bucket_b by segmented running sums
//                  and a quad fan-in tree (msm_reduce.cuh).
//  7. combine      result = sum_w 2^(c*w) * S_w by Horner (host tail, or
//                  k_combine_quad on the device), converted to the
//                  reference's homogeneous projective output.
//
// Packed base records (written once by k_pack_*): affine x, y in Montgomery
// form as 32-bit limbs, then an infinity word; 128 B per G1 point and 256 B
// per G2 point so that every record is one or two whole cache lines and is
// read with 16-byte vector loads.
#pragma once
#include <cstdint>

#include "xyzz.cuh"

namespace gm {

template <class F>
struct Rec;
template <>
struct Rec<Fp> {
  static constexpr int U4 = 8;  // 128 B
};
template <>
struct Rec<Fp2> {
  static constexpr int U4 = 16;  // 256 B
};

// Arithmetic policy with the field product out of line (same data types).
template <class F>
struct OutOfLine;
template <>
struct OutOfLine<Fp> {
  using type = FpOut;
};
template <>
struct OutOfLine<Fp2> {
  using type = Fp2Call;
};

// Policy of the accumulation loop (one out-of-line product only).
template <class F>
struct AccPolicy;
// G1: the integer CIOS product out of line, squares through it too (one
// product function in the loop).
template <>
struct AccPolicy<Fp> {
  using type = FpOutMulOnly;
};
// G2: the whole Fp2 product out of line.  Inlined Karatsuba sums around 30
// Fp calls made the loop overflow the instruction cache (ncu: 9.9% of warp
// samples stalled on instruction fetch against 1.2% for G1); measured
// 12.35 ms against 14.76 ms for the G2 2^18 accumulation.
template <>
struct AccPolicy<Fp2> {
  using type = Fp2Call;
};

template <class A, class B>
GM_DEVI xyzz_t<A> as_xyzz(const xyzz_t<B> &p) {
  return xyzz_t<A>{p.X, p.Y, p.ZZ, p.ZZZ};
}

template <class F>
GM_DEVI uint32_t &limb_ref(typename F::T &a, int i);
template <>
GM_DEVI uint32_t &limb_ref<Fp>(fp_t &a, int i) {
  return a.v[i];
}
template <>
GM_DEVI uint32_t &limb_ref<Fp2>(fp2_t &a, int i) {
  return i < NL ? a.c0.v[i] : a.c1.v[i - NL];
}

// Load x, y of a packed record with 16-byte loads through the read-only path.
template <class F>
GM_DEVI void load_base(typename F::T &x, typename F::T &y, const uint4 *rec) {
  constexpr int L = F::LIMBS;  // 32-bit words per coordinate
#pragma unroll
  for (int q = 0; q < L / 2; q++) {
    const uint4 v = __ldg(rec + q);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int idx = 4 * q + e;
      if (idx < L)
        limb_ref<F>(x, idx) = w[e];
      else
        limb_ref<F>(y, idx - L) = w[e];
    }
  }
}

// Store x, y and the infinity word as one packed record (pad words zero).
template <class F>
GM_DEVI void store_base(uint4 *dst, typename F::T &x, typename F::T &y, uint32_t inf) {
  constexpr int L = F::LIMBS;
  uint32_t w[4 * Rec<F>::U4];
#pragma unroll
  for (int k = 0; k < 4 * Rec<F>::U4; k++) w[k] = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    w[k] = limb_ref<F>(x, k);
    w[L + k] = limb_ref<F>(y, k);
  }
  w[2 * L] = inf;
#pragma unroll
  for (int q = 0; q < Rec<F>::U4; q++) dst[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

GM_DEVI uint32_t base_is_inf(const uint4 *rec, int u4_per_rec, int limbs) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(rec);
  return __ldg(w + 2 * limbs);
}

// Element in the reference layout (u64 limbs, 7 per Fp) <-> registers
template <class F>
GM_DEVI void load_ref(typename F::T &r, const uint64_t *src) {
#pragma unroll
  for (int i = 0; i < F::LIMBS / 2; i++) {
    const uint64_t w = src[i];
    limb_ref<F>(r, 2 * i) = (uint32_t)w;
    limb_ref<F>(r, 2 * i + 1) = (uint32_t)(w >> 32);
  }
}
template <class F>
GM_DEVI void store_ref(uint64_t *dst, typename F::T &a) {
#pragma unroll
  for (int i = 0; i < F::LIMBS / 2; i++)
    dst[i] = (uint64_t)limb_ref<F>(a, 2 * i) | ((uint64_t)limb_ref<F>(a, 2 * i + 1) << 32);
}

// to-Montgomery for either field
template <class F>
GM_DEVI typename F::T field_to_mont(const typename F::T &a);
template <>
GM_DEVI fp_t field_to_mont<Fp>(const fp_t &a) {
  return Fp::to_mont(a);
}
template <>
GM_DEVI fp2_t field_to_mont<Fp2>(const fp2_t &a) {
  return fp2_t{Fp::to_mont(a.c0), Fp::to_mont(a.c1)};
}
template <class F>
GM_DEVI typename F::T field_from_mont(const typename F::T &a);
template <>
GM_DEVI fp_t field_from_mont<Fp>(const fp_t &a) {
  return Fp::from_mont(a);
}
template <>
GM_DEVI fp2_t field_from_mont<Fp2>(const fp2_t &a) {
  return fp2_t{Fp::from_mont(a.c0), Fp::from_mont(a.c1)};
}

// ---------------------------------------------------------------------------
// 0. packing: reference affine structs -> packed records
//    ref_stride_u64: 15 (G1Point, 120 B) or 29 (G2Point, 232 B); the
//    infinity bool sits right after the coordinates.
// ---------------------------------------------------------------------------
template <class F>
__global__ void k_pack_ref(uint4 *__restrict__ out, const uint64_t *__restrict__ pts, int64_t n,
                           int ref_stride_u64, int to_mont) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  constexpr int L = F::LIMBS;
  const uint64_t *src = pts + i * ref_stride_u64;
  const uint8_t inf = reinterpret_cast<const uint8_t *>(src + L)[0];
  typename F::T x, y;
  load_ref<F>(x, src);
  load_ref<F>(y, src + L / 2);
  if (inf) {
    x = F::zero();
    y = F::zero();
  } else if (to_mont) {
    x = field_to_mont<F>(x);
    y = field_to_mont<F>(y);
  }
  store_base<F>(out + i * Rec<F>::U4, x, y, inf ? 1u : 0u);
}

// Fixed-base window table of a resident base set: record (w, i) at index
// w*n + i holds 2^(c w) P_i in affine Montgomery form (w = 0 is P_i), so an
// MSM over the set needs one bucket set for all windows and no window
// doublings.  One thread per point: c XYZZ doublings per window, then the
// affine conversion with one field inversion.
template <class F>
__global__ void __launch_bounds__(128) k_window_table(const uint4 *__restrict__ packed, int64_t n, int c, int W,
                                                      uint4 *__restrict__ table) {
  using FA = typename OutOfLine<F>::type;
  using T = typename F::T;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4 *rec = packed + i * Rec<F>::U4;
  T x, y;
  load_base<F>(x, y, rec);
  if (base_is_inf(rec, Rec<F>::U4, F::LIMBS)) {
    for (int w = 0; w < W; w++) store_base<F>(table + ((int64_t)w * n + i) * Rec<F>::U4, x, y, 1u);
    return;
  }
  store_base<F>(table + i * Rec<F>::U4, x, y, 0u);
  xyzz_t<FA> acc;
  acc.X = x;
  acc.Y = y;
  acc.ZZ = F::one();
  acc.ZZZ = F::one();
  for (int w = 1; w < W; w++) {
    for (int k = 0; k < c; k++) xyzz_dbl_cold<FA>(acc);
    uint4 *dst = table + ((int64_t)w * n + i) * Rec<F>::U4;
    if (xyzz_is_inf(acc)) {
      T z = F::zero();
      store_base<F>(dst, z, z, 1u);
      continue;
    }
    const T I = F::inv(FA::mul(acc.ZZ, acc.ZZZ));
    T ax = FA::mul(acc.X, FA::mul(I, acc.ZZZ));
    T ay = FA::mul(acc.Y, FA::mul(I, acc.ZZ));
    store_base<F>(dst, ax, ay, 0u);
  }
}

// ---------------------------------------------------------------------------
// 1/3. digit decomposition
// ---------------------------------------------------------------------------
constexpr int MAX_SCALAR_LIMBS = 8;

struct DigitParams {
  int c;       // window width in bits
  int W;       // number of windows
  int B;       // buckets per window = 2^(c-1)
  int limbs;   // u64 limbs per scalar
};

// ---------------------------------------------------------------------------
// 2. exclusive scan (three kernels, 1024 elements per block)
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_PER_THREAD = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

GM_DEVI uint32_t block_exclusive_scan(uint32_t v, uint32_t &total) {
  __shared__ uint32_t warp_sums[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < SCAN_THREADS / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  const uint32_t warp_prefix = wid > 0 ? warp_sums[wid - 1] : 0;
  total = warp_sums[SCAN_THREADS / 32 - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

static __global__ void k_scan_blocksum(const uint32_t *__restrict__ in, int64_t K, uint32_t *__restrict__ bsum) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER_THREAD;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++)
    if (base + k < K) s += in[base + k];
  uint32_t total;
  block_exclusive_scan(s, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// single block: exclusive scan of nb block sums in place
static __global__ void k_scan_top(uint32_t *__restrict__ bsum, int nb) {
  uint32_t running = 0;
  for (int base = 0; base < nb; base += SCAN_TILE) {
    const int i0 = base + threadIdx.x * SCAN_PER_THREAD;
    uint32_t v[SCAN_PER_THREAD], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++) {
      v[k] = (i0 + k < nb) ? bsum[i0 + k] : 0;
      s += v[k];
    }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(s, total) + running;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; k++) {
      if (i0 + k < nb) bsum[i0 + k] = ex;
      ex += v[k];
    }
    running += total;
    __syncthreads();
  }
}

static __global__ void k_scan_final(const uint32_t *__restrict__ in, int64_t K, const uint32_t *__restrict__ bsum,
                             uint32_t *__restrict__ out) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER_THREAD;
  uint32_t v[SCAN_PER_THREAD], s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    v[k] = (base + k < K) ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, total) + bsum[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; k++) {
    if (base + k < K) out[base + k] = ex;
    if (base + k == K - 1) out[K] = ex + v[k];
    ex += v[k];
  }
}

// ---------------------------------------------------------------------------
// 4. bucket accumulation over equal slices of the sorted entries
// ---------------------------------------------------------------------------
GM_DEVI int64_t bucket_of(const uint32_t *__restrict__ offsets, int64_t K, uint32_t pos) {
  // largest k in [0, K) with offsets[k] <= pos
  int64_t lo = 0, hi = K;  // offsets[K] > pos
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(offsets + mid) <= pos)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Asynchronous 16-byte global -> shared copy (cp.async, L2 only).
GM_DEVI void cp_async16(void *smem, const void *gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem));
}
GM_DEVI void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
GM_DEVI void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

constexpr int ACC_THREADS = 128;
template <class F>
constexpr int acc_smem_bytes() {
  return 2 * (F::LIMBS / 2) * ACC_THREADS * 16;
}

// An affine base held in the accumulation kernel's shared-memory stage
// ([chunk][thread] uint4 layout), read word by word at first use; y is
// negated for a negative digit.
template <class F, int CH>
struct StagedPoint {
  const uint4 (*rec)[ACC_THREADS];
  int tid;
  bool negate;
  GM_DEVI typename F::T x() const {
    typename F::T r;
#pragma unroll
    for (int k = 0; k < F::LIMBS; k++) {
      const uint4 v = rec[k >> 2][tid];
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
      limb_ref<F>(r, k) = w[k & 3];
    }
    return r;
  }
  // packed records of the point at infinity hold x = y = 0, which is not a
  // curve point (b != 0)
  GM_DEVI bool is_inf() const {
    uint32_t o = 0;
#pragma unroll
    for (int q = 0; q < F::LIMBS / 2; q++) {
      const uint4 v = rec[q][tid];
      o |= v.x | v.y | v.z | v.w;
    }
    return o == 0;
  }
  GM_DEVI typename F::T y() const {
    typename F::T r;
#pragma unroll
    for (int k = 0; k < F::LIMBS; k++) {
      const int idx = F::LIMBS + k;
      const uint4 v = rec[idx >> 2][tid];
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
      limb_ref<F>(r, k) = w[idx & 3];
    }
    return negate ? F::neg(r) : r;
  }
};

// The base of the next entry is staged into shared memory with cp.async while
// the current mixed addition runs, so the random 112/224-byte gather is off
// the critical path.  Each thread owns two slots (double buffer); slots are
// laid out chunk-major ([slot][chunk][thread]) so a warp's 16-byte accesses
// hit consecutive banks.  Only the owning thread reads its slots, so no
// block-level barrier is needed.
// One accumulation slice t of nthreads equal slices of the sorted entries
// (its stage: this thread's two shared-memory slots).
template <class F, int CH>
GM_DEVI void acc_slice(const uint4 *__restrict__ bases, const uint32_t *__restrict__ entries,
                       const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads, int64_t t,
                       xyzz_t<F> *__restrict__ buckets, xyzz_t<F> *__restrict__ part_head,
                       xyzz_t<F> *__restrict__ part_tail, int32_t *__restrict__ head_key,
                       int32_t *__restrict__ tail_key, uint4 (*stage)[CH][ACC_THREADS], int tid) {
  using FA = typename AccPolicy<F>::type;
  int32_t hk = -1, tk = -1;
  // slice length from the actual number of entries (offsets[K])
  const uint32_t M = __ldg(offsets + K);
  const uint64_t chunk64 = ((uint64_t)M + nthreads - 1) / nthreads;
  const uint32_t chunk = chunk64 > 0 ? (uint32_t)chunk64 : 1u;
  const uint64_t start64 = (uint64_t)t * chunk;
  if (start64 < M) {
    const uint32_t start = (uint32_t)start64;
    const uint32_t end = (uint32_t)(start64 + chunk < M ? start64 + chunk : M);
    int64_t k = bucket_of(offsets, K, start);
    uint32_t bend = __ldg(offsets + k + 1);
    bool owns = __ldg(offsets + k) == start;
    xyzz_t<FA> acc;
    xyzz_set_inf(acc);
    uint32_t pos = start;
    uint32_t e_cur = __ldg(entries + pos);
    uint32_t e_nxt = (pos + 1 < end) ? __ldg(entries + pos + 1) : 0u;
    {
      const uint4 *src = bases + (size_t)(e_cur >> 1) * Rec<F>::U4;
#pragma unroll
      for (int q = 0; q < CH; q++) cp_async16(&stage[0][q][tid], src + q);
      cp_async_commit();
    }
    int slot = 0;
    while (true) {
      // prefetch the base of the next entry, and the entry after it
      if (pos + 1 < end) {
        const uint4 *src = bases + (size_t)(e_nxt >> 1) * Rec<F>::U4;
#pragma unroll
        for (int q = 0; q < CH; q++) cp_async16(&stage[slot ^ 1][q][tid], src + q);
      }
      cp_async_commit();
      const uint32_t e_after = (pos + 2 < end) ? __ldg(entries + pos + 2) : 0u;
      cp_async_wait_prev();
      {
        const StagedPoint<F, CH> pt{stage[slot], tid, (e_cur & 1u) != 0};
        if (!pt.is_inf()) xyzz_madd_pt<FA>(acc, pt);
      }
      pos++;
      slot ^= 1;
      e_cur = e_nxt;
      e_nxt = e_after;
      if (pos == bend || pos == end) {
        if (!owns) {
          part_head[t] = as_xyzz<F>(acc);
          hk = (int32_t)k;
        } else if (pos == bend) {
          buckets[k] = as_xyzz<F>(acc);
        } else {
          part_tail[t] = as_xyzz<F>(acc);
          tk = (int32_t)k;
        }
        if (pos == end) break;
        k++;
        while (__ldg(offsets + k + 1) <= pos) k++;
        bend = __ldg(offsets + k + 1);
        owns = true;
        xyzz_set_inf(acc);
      }
    }
  }
  head_key[t] = hk;
  tail_key[t] = tk;
}

// The base of the next entry is staged into shared memory with cp.async while
// the current mixed addition runs, so the random 112/224-byte gather is off
// the critical path.  Each thread owns two slots (double buffer); slots are
// laid out chunk-major ([slot][chunk][thread]) so a warp's 16-byte accesses
// hit consecutive banks.  Only the owning thread reads its slots, so no
// block-level barrier is needed.
template <class F>
__global__ void __launch_bounds__(ACC_THREADS) k_accumulate(const uint4 *__restrict__ bases, const uint32_t *__restrict__ entries,
                                                    const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads,
                                                    xyzz_t<F> *__restrict__ buckets,
                                                    xyzz_t<F> *__restrict__ part_head, xyzz_t<F> *__restrict__ part_tail,
                                                    int32_t *__restrict__ head_key, int32_t *__restrict__ tail_key) {
  constexpr int CH = F::LIMBS / 2;  // 16-byte chunks of x || y
  extern __shared__ uint4 stage_mem[];  // [2][CH][ACC_THREADS], acc_smem_bytes<F>()
  auto stage = reinterpret_cast<uint4(*)[CH][ACC_THREADS]>(stage_mem);
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthreads) return;
  acc_slice<F, CH>(bases, entries, offsets, K, nthreads, t, buckets, part_head, part_tail, head_key, tail_key, stage,
                   threadIdx.x);
}

// One class of a batch in the queued accumulation: its slicing (nthreads
// equal slices, a multiple of 32) and buffers, and its first work item.
template <class F>
struct AccClass {
  const uint4 *bases;
  const uint32_t *entries, *offsets;
  int64_t K, nthreads;
  xyzz_t<F> *buckets, *head, *tail;
  int32_t *hk, *tk;
  int64_t item_first;
};

// Accumulation of every class of a batch in one persistent launch (one
// resident wave) over a device work queue: a work item is 32 consecutive
// slices of one class, taken by a warp from the counter *queue (zero on
// entry); the slicing and outputs are those of k_accumulate, class by class,
// so the fix-up and reduction of each class follow unchanged.
template <class F>
__global__ void __launch_bounds__(ACC_THREADS) k_accumulate_queue(const AccClass<F> *__restrict__ cls, int ncls,
                                                                  int64_t items, uint32_t *__restrict__ queue) {
  constexpr int CH = F::LIMBS / 2;
  extern __shared__ uint4 stage_mem[];
  auto stage = reinterpret_cast<uint4(*)[CH][ACC_THREADS]>(stage_mem);
  const int lane = threadIdx.x & 31;
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(queue, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if ((int64_t)item >= items) break;
    int lo = 0, hi = ncls;  // cls[lo].item_first <= item < cls[hi].item_first
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (cls[mid].item_first <= (int64_t)item)
        lo = mid;
      else
        hi = mid;
    }
    const AccClass<F> c = cls[lo];
    const int64_t t = ((int64_t)item - c.item_first) * 32 + lane;
    acc_slice<F, CH>(c.bases, c.entries, c.offsets, c.K, c.nthreads, t, c.buckets, c.head, c.tail, c.hk, c.tk, stage,
                     threadIdx.x);
    // the next item reuses this thread's stage slots
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
  }
}

}  // namespace gm
