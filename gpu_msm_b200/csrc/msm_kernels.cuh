// Pippenger bucket-method kernels for BLS12-446 G1/G2 on sm_100a.
//
// Pipeline for one MSM  sum_i k_i * P_i  (replaces the per-window host loop of
// pdroalves/gpu_msm src/curve.cu:2538-2677 and the affine multi-limb path
// src/curve.cu:2763-2820):
//
//  1. k_count      signed c-bit digit decomposition of every scalar; count the
//                  non-zero digits per global bucket key  key = w*B + |d|-1
//                  (B = 2^(c-1) buckets per window).
//  2. k_scan_*     exclusive prefix sum of the counts -> bucket offsets.
//  3. k_scatter    counting-sort scatter: the (point, sign) entries land
//                  grouped by bucket key (one radix pass over all windows).
//  4. k_accumulate every thread sums an equal-length slice of the sorted
//                  entries with XYZZ mixed additions; buckets that fit in a
//                  slice are written directly, the edge pieces of buckets that
//                  straddle slices are written as partials.
//  5. k_fixup      the slice that opened a straddling bucket adds the
//                  partials of the following slices.
//  6. k_reduce     per window, sum_b b*Bucket_b by segmented running sums,
//                  applied level by level until one (R, A) pair per window
//                  remains; the window sum is R + A.
//  7. k_combine    result = sum_w 2^(c*w) * S_w by Horner, converted to the
//                  reference's homogeneous projective output.
//
// Packed base records (written once by k_pack_*): affine x, y in Montgomery
// form as 32-bit limbs, then an infinity word; 128 B per G1 point and 256 B
// per G2 point so that every record is one or two whole cache lines and is
// read with 16-byte vector loads.
#pragma once
#include <cstdint>

#include "field_f64.cuh"
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
// Build switch: Fp products of the reduction kernels on the FP64 pipe
// (field_f64.cuh).  Off by default -- the path stays on integer instructions;
// on, the G1 2^20 reduction measured 1.91 ms against 2.03 ms.
#ifndef GM_OOL_F64
#define GM_OOL_F64 0
#endif
template <>
struct OutOfLine<Fp> {
#if GM_OOL_F64
  using type = FpOutF64;
#else
  using type = FpOut;
#endif
};
// G2 keeps the integer product: with its three Fp products on the FP64 pipe
// the G2 2^18 reduction measured 3.01 ms against 2.98 ms.
template <>
struct OutOfLine<Fp2> {
  using type = Fp2Call;
};

// Policy of the accumulation loop (one out-of-line product only).
template <class F>
struct AccPolicy;
// G1 accumulation product: the integer CIOS product by default.  The
// FP64-pipe product (field_f64.cuh, bit-identical) is chosen at run time
// instead when set_fp64_products(true) -- see AccSel below; GM_ACC_F64 sets
// that mode's initial value.  Measured on B200 for the G1 2^20 accumulation:
// 11.10 ms with FP64-pipe products against 13.28 ms.  (Inside the G2 Fp2
// product it measured 12.21 ms against 12.02 ms, so G2 has no FP64 mode.)
#ifndef GM_ACC_F64
#define GM_ACC_F64 0
#endif
// One product function only: squares on the integer pipe beside FP64-pipe
// products (two out-of-line functions in the loop) measured 15.12 ms.
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

// Accumulation policy for the run-time product mode: FP64-pipe products for
// G1 when FP64 is set, else AccPolicy's.
template <class F, bool FP64>
struct AccSel {
  using type = typename AccPolicy<F>::type;
};
template <>
struct AccSel<Fp, true> {
  using type = FpOutF64;
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

GM_DEVI uint32_t window_bits(const uint64_t s[MAX_SCALAR_LIMBS], int limbs, int off, int c) {
  const int l = off >> 6, sh = off & 63;
  if (l >= limbs) return 0;
  uint64_t v = s[l] >> sh;
  if (sh + c > 64 && l + 1 < limbs) v |= s[l + 1] << (64 - sh);
  return (uint32_t)(v & ((1ull << c) - 1));
}

// Calls fn(w, d) for every non-zero signed digit d of the scalar, where
// scalar = sum_w d_w 2^(c w) and |d_w| <= 2^(c-1).
template <class Fn>
GM_DEVI void for_each_digit(const uint64_t *__restrict__ scalar, const DigitParams &dp, Fn fn) {
  uint64_t s[MAX_SCALAR_LIMBS];
#pragma unroll
  for (int l = 0; l < MAX_SCALAR_LIMBS; l++) s[l] = l < dp.limbs ? scalar[l] : 0;
  uint32_t carry = 0;
  for (int w = 0; w < dp.W; w++) {
    const uint32_t v = window_bits(s, dp.limbs, w * dp.c, dp.c) + carry;
    int d;
    if (v > (uint32_t)dp.B) {
      d = (int)v - 2 * dp.B;
      carry = 1;
    } else {
      d = (int)v;
      carry = 0;
    }
    if (d != 0) fn(w, d);
  }
}

// The sort reads only the scalars: entries of bases at infinity are sorted
// like any other and skipped by the accumulation.
static __global__ void k_count(const uint64_t *__restrict__ scalars, int64_t n, DigitParams dp,
                               uint32_t *__restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for_each_digit(scalars + i * dp.limbs, dp, [&](int w, int d) {
    const int b = (d < 0 ? -d : d) - 1;
    atomicAdd(&counts[w * dp.B + b], 1u);
  });
}

// Consumes counts back down to zero; entry = (point index << 1) | negative.
static __global__ void k_scatter(const uint64_t *__restrict__ scalars, int64_t n, DigitParams dp,
                                 const uint32_t *__restrict__ offsets, uint32_t *__restrict__ counts,
                                 uint32_t *__restrict__ entries) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for_each_digit(scalars + i * dp.limbs, dp, [&](int w, int d) {
    const int key = w * dp.B + (d < 0 ? -d : d) - 1;
    const uint32_t rank = atomicSub(&counts[key], 1u) - 1u;
    entries[offsets[key] + rank] = ((uint32_t)i << 1) | (d < 0 ? 1u : 0u);
  });
}

// Many MSMs in one pipeline (batched mode).  MSM i owns the flattened point
// ids [point_start[i], point_start[i+1]); its j-th point uses base record
// base_off[i] + j of the shared table and scalar row sc_off[i] + j.  Its
// bucket keys are i*W*B + w*B + |d|-1, so one counting sort, one
// accumulation and one reduction serve every MSM of the batch.
// With a fixed-base window table (pc_stride = table points n > 0) the window
// index moves from the bucket key to the base record: keys are i*B + |d|-1
// and the entry addresses record w*n + base of the table.
struct MultiDesc {
  const int64_t *point_start;  // [count + 1]
  const int64_t *base_off;     // [count]
  const int64_t *sc_off;       // [count]
  int count;
};

GM_DEVI int msm_of(const int64_t *__restrict__ ps, int count, int64_t p) {
  int lo = 0, hi = count;  // ps[lo] <= p < ps[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(ps + mid) <= p)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

static __global__ void k_count_multi(const uint64_t *__restrict__ scalars, int64_t P, MultiDesc md, DigitParams dp,
                                     int64_t pc_stride, uint32_t *__restrict__ counts) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int i = msm_of(md.point_start, md.count, p);
  const int64_t j = p - __ldg(md.point_start + i);
  const int64_t bi = __ldg(md.base_off + i) + j;
  const int64_t kbase = (int64_t)i * (pc_stride ? 1 : dp.W) * dp.B;
  for_each_digit(scalars + (__ldg(md.sc_off + i) + j) * dp.limbs, dp, [&](int w, int d) {
    atomicAdd(&counts[kbase + (pc_stride ? 0 : (int64_t)w * dp.B) + (d < 0 ? -d : d) - 1], 1u);
  });
}

static __global__ void k_scatter_multi(const uint64_t *__restrict__ scalars, int64_t P, MultiDesc md,
                                       DigitParams dp, int64_t pc_stride, const uint32_t *__restrict__ offsets,
                                       uint32_t *__restrict__ counts, uint32_t *__restrict__ entries) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int i = msm_of(md.point_start, md.count, p);
  const int64_t j = p - __ldg(md.point_start + i);
  const int64_t bi = __ldg(md.base_off + i) + j;
  const int64_t kbase = (int64_t)i * (pc_stride ? 1 : dp.W) * dp.B;
  for_each_digit(scalars + (__ldg(md.sc_off + i) + j) * dp.limbs, dp, [&](int w, int d) {
    const int64_t key = kbase + (pc_stride ? 0 : (int64_t)w * dp.B) + (d < 0 ? -d : d) - 1;
    const uint32_t rank = atomicSub(&counts[key], 1u) - 1u;
    const int64_t rec = pc_stride ? (int64_t)w * pc_stride + bi : bi;
    entries[offsets[key] + rank] = ((uint32_t)rec << 1) | (d < 0 ? 1u : 0u);
  });
}

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
template <class F, bool FP64 = false>
__global__ void __launch_bounds__(ACC_THREADS) k_accumulate(const uint4 *__restrict__ bases, const uint32_t *__restrict__ entries,
                                                    const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads,
                                                    xyzz_t<F> *__restrict__ buckets,
                                                    xyzz_t<F> *__restrict__ part_head, xyzz_t<F> *__restrict__ part_tail,
                                                    int32_t *__restrict__ head_key, int32_t *__restrict__ tail_key) {
  using T = typename F::T;
  using FA = typename AccSel<F, FP64>::type;
  constexpr int CH = F::LIMBS / 2;  // 16-byte chunks of x || y
  extern __shared__ uint4 stage_mem[];  // [2][CH][ACC_THREADS], acc_smem_bytes<F>()
  auto stage = reinterpret_cast<uint4(*)[CH][ACC_THREADS]>(stage_mem);
  const int tid = threadIdx.x;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthreads) return;
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

// 5. the slice that opened a straddling bucket folds in the following slices
template <class F>
__global__ void __launch_bounds__(128) k_fixup(const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads,
                                               xyzz_t<F> *__restrict__ buckets, const xyzz_t<F> *__restrict__ part_head,
                                               const xyzz_t<F> *__restrict__ part_tail,
                                               const int32_t *__restrict__ head_key, const int32_t *__restrict__ tail_key,
                                               uint32_t *__restrict__ err) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthreads) return;
  const int32_t k = tail_key[t];
  if (k < 0) return;
  const uint32_t M = __ldg(offsets + K);
  const uint64_t chunk64 = ((uint64_t)M + nthreads - 1) / nthreads;
  const uint32_t chunk = chunk64 > 0 ? (uint32_t)chunk64 : 1u;
  using FA = typename OutOfLine<F>::type;
  xyzz_t<FA> acc = as_xyzz<FA>(part_tail[t]);
  const uint64_t bend = __ldg(offsets + k + 1);
  int64_t t2 = t + 1;
  while (t2 < nthreads) {
    if (head_key[t2] != k) {  // cannot happen for a consistent slicing
      atomicOr(err, 1u);
      break;
    }
    xyzz_add_cold<FA>(acc, as_xyzz<FA>(part_head[t2]));
    if ((uint64_t)(t2 + 1) * chunk >= bend) break;
    t2++;
  }
  buckets[k] = as_xyzz<F>(acc);
}

// ---------------------------------------------------------------------------
// 6. bucket reduction: per window  S = sum_{j=0}^{B-1} (j+1) * V_j.
//
// k_reduce_segments: one thread per segment [j0, j0+L) of a window computes,
// by a running sum from the top, ws = sum (j - j0) V_j and a = sum V_j, then
// its share of S directly:  ws + (j0 + 1) * a  (double-and-add by the small
// integer j0 + 1).  The segment shares of a window are then added by a
// fan-in tree (k_tree_sum).  Serial depth: 2L additions + log2(B) doublings
// + log_fan(B/L) tree levels, with every stage spread over all segments.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(128) k_reduce_segments(const xyzz_t<F> *__restrict__ buckets,
                                                         const uint32_t *__restrict__ offsets, int W, int B, int L,
                                                         xyzz_t<F> *__restrict__ V_out) {
  using FA = typename OutOfLine<F>::type;
  const int nseg = (B + L - 1) / L;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)W * nseg) return;
  const int w = (int)(t / nseg), s = (int)(t % nseg);
  const int64_t kb = (int64_t)w * B;
  xyzz_t<FA> acc, ws;
  xyzz_set_inf(acc);
  xyzz_set_inf(ws);
  const int j0 = s * L, j1 = min(B, j0 + L);
  for (int j = j1 - 1; j >= j0; j--) {
    if (__ldg(offsets + kb + j + 1) != __ldg(offsets + kb + j)) xyzz_add<FA>(acc, as_xyzz<FA>(buckets[kb + j]));
    if (j > j0) xyzz_add<FA>(ws, acc);
  }
  // ws += (j0 + 1) * acc, MSB-first double-and-add
  const uint32_t mult = (uint32_t)j0 + 1u;
  if (!xyzz_is_inf(acc)) {
    xyzz_t<FA> m;
    xyzz_set_inf(m);
    for (int b = 31 - __clz(mult); b >= 0; b--) {
      xyzz_dbl<FA>(m, m);
      if ((mult >> b) & 1u) xyzz_add<FA>(m, acc);
    }
    xyzz_add<FA>(ws, m);
  }
  V_out[t] = as_xyzz<F>(ws);
}

// out[g][i] = sum_{k < fan} in[g][i*fan + k]  (groups of N elements)
template <class F>
__global__ void __launch_bounds__(128) k_tree_sum(const xyzz_t<F> *__restrict__ in, int groups, int N, int fan,
                                                  xyzz_t<F> *__restrict__ out) {
  using FA = typename OutOfLine<F>::type;
  const int nout = (N + fan - 1) / fan;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)groups * nout) return;
  const int g = (int)(t / nout), i = (int)(t % nout);
  const int64_t base = (int64_t)g * N + (int64_t)i * fan;
  xyzz_t<FA> acc = as_xyzz<FA>(in[base]);
  for (int k = 1; k < fan && i * fan + k < N; k++) xyzz_add<FA>(acc, as_xyzz<FA>(in[base + k]));
  out[t] = as_xyzz<F>(acc);
}

// 7. Horner over windows on the device, one thread per MSM (used inside
// CUDA-graph capture and for batches, where the host tail is not used);
// writes the homogeneous projective result (X, Y, Z; u64 limbs; Montgomery).
template <class F>
__global__ void k_combine(const xyzz_t<F> *__restrict__ S, int n_msm, int W, int c, uint64_t *__restrict__ out_proj) {
  using FA = typename OutOfLine<F>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_msm) return;
  xyzz_t<FA> res;
  xyzz_set_inf(res);
  for (int w = W - 1; w >= 0; w--) {
    if (!xyzz_is_inf(res))
      for (int k = 0; k < c; k++) xyzz_dbl<FA>(res, res);
    xyzz_add<FA>(res, as_xyzz<FA>(S[(int64_t)i * W + w]));
  }
  typename F::T X, Y, Z;
  xyzz_to_proj<FA>(X, Y, Z, res);
  constexpr int H = F::LIMBS / 2;  // u64 words per coordinate
  uint64_t *o = out_proj + (int64_t)i * 3 * H;
  store_ref<F>(o, X);
  store_ref<F>(o + H, Y);
  store_ref<F>(o + 2 * H, Z);
}

// Horner per MSM of a batch; MSM i writes result slot out_index[i].
template <class F>
__global__ void k_combine_indexed(const xyzz_t<F> *__restrict__ S, int n_msm, int W, int c,
                                  const int32_t *__restrict__ out_index, uint64_t *__restrict__ out_proj) {
  using FA = typename OutOfLine<F>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_msm) return;
  xyzz_t<FA> res;
  xyzz_set_inf(res);
  for (int w = W - 1; w >= 0; w--) {
    if (!xyzz_is_inf(res))
      for (int k = 0; k < c; k++) xyzz_dbl<FA>(res, res);
    xyzz_add<FA>(res, as_xyzz<FA>(S[(int64_t)i * W + w]));
  }
  typename F::T X, Y, Z;
  xyzz_to_proj<FA>(X, Y, Z, res);
  constexpr int H = F::LIMBS / 2;
  uint64_t *o = out_proj + (int64_t)__ldg(out_index + i) * 3 * H;
  store_ref<F>(o, X);
  store_ref<F>(o + H, Y);
  store_ref<F>(o + 2 * H, Z);
}

}  // namespace gm
