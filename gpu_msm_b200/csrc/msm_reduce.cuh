// Bucket reduction, long-run fix-up and window combination for the MSM
// pipelines (single and batched).
//
// Bucket reduction.  Per window (group g of G) with B buckets V_0..V_{B-1}:
//     S_g = sum_j (j + 1) V_j.
// Level 0 cuts the buckets into segments of L0 and computes in one thread per
// segment, by a running sum from the top,
//     T_s = sum_r (r + 1) V_{s L0 + r},   A_s = sum_r V_{s L0 + r},
// two additions per bucket and nothing else.  Then
//     S_g = sum_s T_s + L0 * sum_s s A_s.
// Level 1 cuts the A_s into segments of L1; a cooperative group of lanes
// (coop.cuh) per segment s' computes  D = sum_r r A_{s' L1 + r},  A' = sum_r A_{s' L1 + r}  and
//     E_{s'} = L0 * (D + (s' L1) A')          (double-and-add, then doublings)
// so that  sum_s s A_s = sum_{s'} (D + s' L1 A')  and
//     S_g = sum_s T_s + sum_{s'} E_{s'}.
// A cooperative fan-in tree adds the nseg0 + nseg1 values of every group.
// Level 0 is throughput-bound (it holds nearly all the work and enough
// threads to fill the GPU); the few, serial additions of level 1 and the tree
// run on quads to cut their latency.  This replaces the reference's per-block
// partial buckets and per-window host combine (src/curve.cu:1557-1654,
// :2060-2179) with work that stays on the device.
#pragma once
#include "msm_kernels.cuh"
#include "coop.cuh"

namespace gm {

// Level 0: segments (group, s) in a grid-stride loop.  The host picks L0 so
// that all segments fit in one resident wave when it can (no partial second
// wave doubling the serial time).  X has M values per group; T_s goes to
// X[g*M + s], A_s to A0[g*nseg0 + s].  Empty buckets (equal offsets) are not
// read; an empty segment costs two stores.
template <class F>
__global__ void __launch_bounds__(128) k_red_level0(const xyzz_t<F> *__restrict__ buckets,
                                                       const uint32_t *__restrict__ offsets, int64_t G, int B, int L0,
                                                       int nseg0, xyzz_t<F> *__restrict__ X, int M,
                                                       xyzz_t<F> *__restrict__ A0) {
  using FA = typename OutOfLine<F>::type;
  const int64_t total = G * nseg0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int64_t g = t / nseg0;
    const int s = (int)(t % nseg0);
    const int64_t kb = g * B;
    xyzz_t<FA> acc, ws;
    xyzz_set_inf(acc);
    xyzz_set_inf(ws);
    const int j0 = s * L0, j1 = min(B, j0 + L0);
    if (__ldg(offsets + kb + j0) != __ldg(offsets + kb + j1)) {  // any entries in the segment
      for (int j = j1 - 1; j >= j0; j--) {
        if constexpr (sizeof(typename F::T) == sizeof(fp_t)) {
          if (__ldg(offsets + kb + j + 1) != __ldg(offsets + kb + j)) xyzz_add<FA>(acc, as_xyzz<FA>(buckets[kb + j]));
          xyzz_add<FA>(ws, acc);
        } else {
          // Fp2: the addition out of line keeps the loop within the register file
          if (__ldg(offsets + kb + j + 1) != __ldg(offsets + kb + j))
            xyzz_add_cold<FA>(acc, as_xyzz<FA>(buckets[kb + j]));
          xyzz_add_cold<FA>(ws, acc);
        }
      }
    }
    X[g * M + s] = as_xyzz<F>(ws);
    A0[g * nseg0 + s] = as_xyzz<F>(acc);
  }
}

// Level 1: one cooperative group of lanes per (group, segment s').  Writes E_{s'} to X[g*M + nseg0 + s'].
template <class F>
__global__ void __launch_bounds__(128) k_red_level1(const xyzz_t<F> *__restrict__ A0, int64_t G, int nseg0, int L1,
                                                    int nseg1, int L0, xyzz_t<F> *__restrict__ X, int M) {
  using C = Coop<F>;
  using FA = typename C::A;
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / C::LANES;
  if (t >= G * nseg1) return;
  const int64_t g = t / nseg1;
  const int s = (int)(t % nseg1);
  const int r0 = s * L1, r1 = min(nseg0, r0 + L1);
  xyzz_t<FA> acc, ws;
  xyzz_set_inf(acc);
  xyzz_set_inf(ws);
  for (int r = r1 - 1; r >= r0; r--) {
    C::add(acc, as_xyzz<FA>(A0[g * nseg0 + r]));
    if (r > r0) C::add(ws, acc);
  }
  // ws = sum (r - r0) A_r; add (s L1) * acc, then scale by L0
  xyzz_t<FA> m;
  coop_mul_small<F>(m, acc, (uint32_t)r0);
  C::add(ws, m);
  coop_mul_small<F>(m, ws, (uint32_t)L0);
  if (coop_leader<F>()) X[g * M + nseg0 + s] = as_xyzz<F>(m);
}

// out[g*nout + i] = sum_{k < fan} in[g*N + i*fan + k], one cooperative
// group per output
template <class F>
__global__ void __launch_bounds__(128) k_tree_quad(const xyzz_t<F> *__restrict__ in, int64_t G, int N, int fan,
                                                   xyzz_t<F> *__restrict__ out) {
  using C = Coop<F>;
  using FA = typename C::A;
  const int nout = (N + fan - 1) / fan;
  const int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / C::LANES;
  if (t >= G * nout) return;
  const int64_t g = t / nout;
  const int i = (int)(t % nout);
  const int64_t base = g * N + (int64_t)i * fan;
  xyzz_t<FA> acc = as_xyzz<FA>(in[base]);
  for (int k = 1; k < fan && i * fan + k < N; k++) C::add(acc, as_xyzz<FA>(in[base + k]));
  if (coop_leader<F>()) out[t] = as_xyzz<F>(acc);
}

// ---------------------------------------------------------------------------
// Fix-up of buckets that straddle accumulation slices.  Slice t0 holds the
// tail piece of bucket k (part_tail[t0]); slices t0+1..t1 hold head pieces
// (part_head).  Runs of at most FIX_SHORT heads are folded serially by the
// owner of the tail; longer runs (a bucket much larger than a slice, e.g. all
// the scalars equal to 1) are queued and folded by k_fixup_long, one block of
// cooperative groups per run with a shared-memory tree.
// ---------------------------------------------------------------------------
constexpr int FIX_SHORT = 8;
constexpr int FIX_LONG_BLOCKS = 64;

// long_q: [0] = count, then bucket keys
template <class F>
__global__ void __launch_bounds__(128) k_fixup_split(const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads,
                                                     xyzz_t<F> *__restrict__ buckets,
                                                     const xyzz_t<F> *__restrict__ part_head,
                                                     const xyzz_t<F> *__restrict__ part_tail,
                                                     const int32_t *__restrict__ head_key,
                                                     const int32_t *__restrict__ tail_key, uint32_t *__restrict__ err,
                                                     int32_t *__restrict__ long_q, int64_t long_cap) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthreads) return;
  const int32_t k = tail_key[t];
  if (k < 0) return;
  const uint32_t M = __ldg(offsets + K);
  const uint64_t chunk64 = ((uint64_t)M + nthreads - 1) / nthreads;
  const uint64_t chunk = chunk64 > 0 ? chunk64 : 1u;
  const uint64_t bend = __ldg(offsets + k + 1);
  const int64_t t1 = (int64_t)((bend - 1) / chunk);  // slice holding the bucket's last entry
  if (t1 - t > FIX_SHORT) {
    const int32_t slot = atomicAdd(long_q, 1);
    if (slot < long_cap)
      long_q[1 + slot] = k;
    else
      atomicOr(err, 2u);
    return;
  }
  using FA = typename OutOfLine<F>::type;
  xyzz_t<FA> acc = as_xyzz<FA>(part_tail[t]);
  for (int64_t t2 = t + 1; t2 <= t1 && t2 < nthreads; t2++) {
    if (head_key[t2] != k) {  // cannot happen for a consistent slicing
      atomicOr(err, 1u);
      break;
    }
    xyzz_add_cold<FA>(acc, as_xyzz<FA>(part_head[t2]));
  }
  buckets[k] = as_xyzz<F>(acc);
}

template <class F>
__global__ void __launch_bounds__(128) k_fixup_long(const uint32_t *__restrict__ offsets, int64_t K, int64_t nthreads,
                                                    xyzz_t<F> *__restrict__ buckets,
                                                    const xyzz_t<F> *__restrict__ part_head,
                                                    const xyzz_t<F> *__restrict__ part_tail,
                                                    const int32_t *__restrict__ head_key, uint32_t *__restrict__ err,
                                                    const int32_t *__restrict__ long_q, int64_t long_cap) {
  using C = Coop<F>;
  using FA = typename C::A;
  constexpr int GROUPS = 128 / C::LANES;  // cooperative groups per block
  __shared__ xyzz_t<F> part[GROUPS];
  const int grp = threadIdx.x / C::LANES;
  const bool leader = coop_leader<F>();
  const int64_t n_long = min((int64_t)long_q[0], long_cap);
  const uint32_t M = __ldg(offsets + K);
  const uint64_t chunk64 = ((uint64_t)M + nthreads - 1) / nthreads;
  const uint64_t chunk = chunk64 > 0 ? chunk64 : 1u;
  for (int64_t item = blockIdx.x; item < n_long; item += gridDim.x) {
    const int32_t k = long_q[1 + item];
    const int64_t t0 = (int64_t)(__ldg(offsets + k) / chunk);
    const int64_t t1 = min((int64_t)((__ldg(offsets + k + 1) - 1) / chunk), nthreads - 1);
    // group j folds run positions j, j+GROUPS, ... (position 0 is the tail piece)
    xyzz_t<FA> acc;
    xyzz_set_inf(acc);
    for (int64_t p = grp; p <= t1 - t0; p += GROUPS) {
      const int64_t ts = t0 + p;
      if (p == 0) {
        C::add(acc, as_xyzz<FA>(part_tail[ts]));
      } else if (head_key[ts] != k) {
        if (leader) atomicOr(err, 1u);
      } else {
        C::add(acc, as_xyzz<FA>(part_head[ts]));
      }
    }
    if (leader) part[grp] = as_xyzz<F>(acc);
    __syncthreads();
    for (int h = GROUPS / 2; h >= 1; h >>= 1) {
      if (grp < h) C::add(acc, as_xyzz<FA>(part[grp + h]));
      __syncthreads();
      if (grp < h && leader) part[grp] = as_xyzz<F>(acc);
      __syncthreads();
    }
    if (threadIdx.x == 0) buckets[k] = part[0];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Window combination on the device, one cooperative group per MSM: result = sum_w
// 2^(c w) S_w by Horner; homogeneous projective output (u64 limbs,
// Montgomery).  out_index (optional) maps MSM i to its result slot.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(128) k_combine_quad(const xyzz_t<F> *__restrict__ S, int n_msm, int W, int c,
                                                      const int32_t *__restrict__ out_index,
                                                      uint64_t *__restrict__ out_proj) {
  using C = Coop<F>;
  using FA = typename C::A;
  const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / C::LANES);
  if (i >= n_msm) return;
  xyzz_t<FA> res;
  xyzz_set_inf(res);
  for (int w = W - 1; w >= 0; w--) {
    if (!xyzz_is_inf(res))
      for (int k = 0; k < c; k++) C::dbl(res);
    C::add(res, as_xyzz<FA>(S[(int64_t)i * W + w]));
  }
  if (!coop_leader<F>()) return;
  typename F::T Xp, Yp, Zp;
  xyzz_to_proj<FA>(Xp, Yp, Zp, res);
  constexpr int H = F::LIMBS / 2;
  const int64_t slot = out_index ? (int64_t)__ldg(out_index + i) : (int64_t)i;
  uint64_t *o = out_proj + slot * 3 * H;
  store_ref<F>(o, Xp);
  store_ref<F>(o + H, Yp);
  store_ref<F>(o + 2 * H, Zp);
}

// ---------------------------------------------------------------------------
// Host side: workspace layout and launch sequence of the reduction.
// ---------------------------------------------------------------------------
struct RedLayout {
  int64_t G = 0;
  int sms = 1, dev = 0;  // device the level-0 grid is sized for
  int B = 0, L0 = 0, nseg0 = 0, L1 = 0, nseg1 = 0, M = 0;
  static constexpr int FAN = 2;
  size_t o_X = 0, o_A0 = 0, o_t[2] = {0, 0};

  // wave_threads: level-0 threads resident at once on the device.  L0 is at
  // least 16 buckets for G1 and 4 for G2 (an Fp2 addition takes three times
  // as long, so G2 wants shorter chains), and larger when the segments would
  // not fit one wave.  coop_wave: threads of the cooperative level-1 kernel
  // resident at once (0: no limit); L1 is at least 4 or 8 segments (below),
  // and larger when the level-1 groups (Coop<F>::LANES threads each) would
  // not fit one wave: a second wave would double the level's serial time.
  template <class F, class Carver>
  void plan(int64_t G_, int B_, int64_t wave_threads, Carver &cv, int64_t coop_wave = 0) {
    G = G_;
    B = B_;
    int64_t l0 = sizeof(typename F::T) == sizeof(fp_t) ? 16 : 4;
    if (wave_threads > 0) l0 = std::max<int64_t>(l0, (G * B + wave_threads - 1) / wave_threads);
    L0 = (int)std::min<int64_t>(l0, B);
    nseg0 = (B + L0 - 1) / L0;
    // 4 segments when the groups of 4-segment runs fill at most half a wave
    // (more and shorter chains; 2^16 MSMs: G2 reduction 2.01 -> 1.75 ms, G1
    // 1.28 -> 1.18 ms), else 8 (with 4 the groups of G1 2^20 / G2 2^18 fill
    // the wave, and their reductions measured 2.05 / 4.45 ms against 2.00 /
    // 3.94 ms)
    int64_t l1 = 8;
    if (coop_wave > 0 && G * nseg0 * Coop<F>::LANES / 4 <= coop_wave / 2) l1 = 4;
    if (coop_wave > 0) l1 = std::max<int64_t>(l1, (G * nseg0 * Coop<F>::LANES + coop_wave - 1) / coop_wave);
    L1 = (int)std::min<int64_t>(l1, nseg0);
    nseg1 = nseg0 > 1 ? (nseg0 + L1 - 1) / L1 : 0;
    M = nseg0 + nseg1;
    o_X = cv.template take<xyzz_t<F>>((size_t)(G * M));
    o_A0 = cv.template take<xyzz_t<F>>((size_t)(G * nseg0));
    const int64_t t1 = G * ((M + FAN - 1) / FAN);
    o_t[0] = cv.template take<xyzz_t<F>>((size_t)std::max<int64_t>(1, t1));
    o_t[1] = cv.template take<xyzz_t<F>>((size_t)std::max<int64_t>(1, (t1 + FAN - 1) / FAN + G));
  }
};

}  // namespace gm
