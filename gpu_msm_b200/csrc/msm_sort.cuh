// Deterministic sort of the (bucket, point) entries of one MSM or of one
// batch class: a stable two-pass radix sort staged through shared memory.
//
// Every scalar k_j of MSM i gives, per window w, a signed c-bit digit d; a
// non-zero digit is an entry (record << 1 | d < 0) in bucket b = |d| - 1 of
// group g (g = i*W + w, or g = i when the set has a fixed-base window table
// and all windows share one bucket set).  The accumulation needs the entries
// grouped by bucket key g*B + b (B = 2^(c-1)) and the bucket offsets.  The
// reference has no sort: its kernels scan all n points for every bucket
// (src/curve.cu:1180-1371, :1659-1728).
//
// Pass A reads the scalars once per tile of SA_THREADS * ppt points (one MSM
// per tile; ppt = 2, 4 or 8 points per thread, chosen per plan),
// staged in shared memory, computes the digits window by window, and
// partitions the entries by (group, hi) where hi = b >> LB: every block
// counts its tile's entries per (group, hi) with shared-memory atomics
// (k_sort_a_count), one exclusive scan over the count matrix
// [group][hi][tile] gives every (group, hi, tile) its output range, and the
// same block reads the digits back (the counting kernel stores them) and
// writes each entry at its range start plus its rank inside the tile
// (k_sort_a_scatter).  Ranks come from
// per-warp counters and a ballot per digit bit over 32 consecutive points,
// so the order inside a (group, hi) range is the point order.
// Pass B (only when c - 1 > 8 bits) sorts every (group, hi) segment by
// lo = b mod 2^LB the same way, over tiles of SB_TILE entries cut along the
// segment boundaries, and stages each tile in shared memory so that its
// writes are contiguous runs.  Both passes are stable, so the entries of one
// bucket end up in point order: the sort and everything after it are
// deterministic (no atomics decide an order).
// Bucket offsets are read off the scanned count matrices (the range start of
// (segment, digit, first tile)); no per-entry global atomic is used anywhere.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "msm_kernels.cuh"

namespace gm {

constexpr int SA_THREADS = 256;
constexpr int SA_PPT = 4;                        // default points per thread (pass A): 2, 4 or 8
constexpr int SA_TP = SA_THREADS * SA_PPT;       // default points per pass-A tile
constexpr int SB_THREADS = 256;
constexpr int SB_IPT = 8;                        // entries per thread (pass B)
constexpr int SB_TILE = SB_THREADS * SB_IPT;     // entries per pass-B tile
constexpr int SORT_WARPS = 8;

// The MSMs of one sort.  A single MSM passes null arrays and n_single.
struct SortDesc {
  const int64_t *point_start = nullptr;  // [count + 1] flattened point ids of each MSM
  const int64_t *base_off = nullptr;     // [count] first base record of each MSM
  const int64_t *sc_off = nullptr;       // [count] first scalar row of each MSM
  const int32_t *tile_first = nullptr;   // [count + 1] first pass-A tile of each MSM
  int count = 1;
  int64_t n_single = 0;                  // points of a single MSM (arrays null)
  int64_t pc_stride = 0;                 // > 0: fixed-base table mode (record w*pc_stride + base)
};

struct SortParams {
  DigitParams dp{};
  int S = 1;        // groups per MSM: W, or 1 in fixed-base table mode
  int passes = 1;
  int HB = 0, LB = 0;
  int RA = 1, RB = 1;  // digit ranges of pass A (hi) and pass B (lo)
  int64_t NS = 0;      // segments (group, hi) of pass B
  int64_t lenA = 0;    // pass-A counters
  int64_t lenB = 0;    // pass-B counters (upper bound)
  int64_t tilesA = 0;
  int64_t tilesB_max = 0;
  int ppt = SA_PPT;          // pass-A points per thread (2, 4 or 8)
  int tp = SA_TP;            // pass-A points per tile (SA_THREADS * ppt)
};

struct TileA {
  int i, t, tiles;
  int64_t p0, np, base_off, sc_row, cbase;
};

GM_DEVI TileA tile_a_info(const SortDesc &sd, const SortParams &sp, int tile) {
  TileA ti;
  if (sd.point_start == nullptr) {
    ti.i = 0;
    ti.t = tile;
    ti.tiles = (int)sp.tilesA;
    ti.p0 = (int64_t)tile * sp.tp;
    ti.np = min((int64_t)sp.tp, sd.n_single - ti.p0);
    ti.base_off = ti.p0;
    ti.sc_row = ti.p0;
    ti.cbase = 0;
    return ti;
  }
  int lo = 0, hi = sd.count;  // tile_first[lo] <= tile < tile_first[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(sd.tile_first + mid) <= tile)
      lo = mid;
    else
      hi = mid;
  }
  const int f0 = __ldg(sd.tile_first + lo);
  ti.i = lo;
  ti.t = tile - f0;
  ti.tiles = __ldg(sd.tile_first + lo + 1) - f0;
  const int64_t ps = __ldg(sd.point_start + lo), pe = __ldg(sd.point_start + lo + 1);
  const int64_t j0 = (int64_t)ti.t * sp.tp;
  ti.p0 = ps + j0;
  ti.np = min((int64_t)sp.tp, pe - ti.p0);
  ti.base_off = __ldg(sd.base_off + lo) + j0;
  ti.sc_row = __ldg(sd.sc_off + lo) + j0;
  ti.cbase = (int64_t)sp.S * sp.RA * f0;
  return ti;
}

// index of the pass-A counter of (MSM tile info, group-in-MSM, hi digit)
GM_DEVI int64_t idx_a(const TileA &ti, const SortParams &sp, int s_local, int d, int t) {
  return ti.cbase + ((int64_t)s_local * sp.RA + d) * ti.tiles + t;
}

GM_DEVI uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Lanes of the warp holding the same bin (a BITS-wide value), by one ballot
// per bit; only meaningful for lanes with valid set.
template <int BITS>
GM_DEVI uint32_t same_bin_lanes(uint32_t bin, bool valid) {
  uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
  for (int k = 0; k < BITS; k++) {
    const uint32_t b = __ballot_sync(0xffffffffu, (bin >> k) & 1u);
    peers &= ((bin >> k) & 1u) ? b : ~b;
  }
  return peers;
}

// Signed digit of window w from staged scalar limbs and the running carry.
GM_DEVI int signed_digit(const uint64_t *s, int limbs, int w, const DigitParams &dp, uint32_t &carry) {
  const int off = w * dp.c, l = off >> 6, sh = off & 63;
  uint64_t v = 0;
  if (l < limbs) {
    v = s[l] >> sh;
    if (sh + dp.c > 64 && l + 1 < limbs) v |= s[l + 1] << (64 - sh);
  }
  const uint32_t raw = (uint32_t)(v & ((1ull << dp.c) - 1)) + carry;
  if (raw > (uint32_t)dp.B) {
    carry = 1;
    return (int)raw - 2 * dp.B;
  }
  carry = 0;
  return (int)raw;
}

// Windows per chunk of the pass-A scatter: its per-warp counters are
// [SORT_WARPS][chunk groups][RA].
constexpr int SA_CHUNK_W = 4;
__host__ __device__ inline int sort_a_chunk(const SortParams &sp) { return sp.dp.W < SA_CHUNK_W ? sp.dp.W : SA_CHUNK_W; }
// counter groups of one chunk: its windows, or the one group of the
// fixed-base table mode
__host__ __device__ inline int sort_a_groups(const SortParams &sp) { return sp.S == 1 ? 1 : sort_a_chunk(sp); }
// scatter blocks per pass-A tile: one per chunk, or one for the single group
// (whose chunks depend on each other's counts)
__host__ __device__ inline int sort_a_blocks_per_tile(const SortParams &sp) {
  return sp.S == 1 ? 1 : (sp.dp.W + sort_a_chunk(sp) - 1) / sort_a_chunk(sp);
}

// Dynamic shared memory of k_sort_a_*: for counting, the staged scalars and
// the counters [S][RA]; for the scatter, the per-warp counters
// [SORT_WARPS][groups][RA] and a running count per hi.
inline size_t sort_a_smem(const SortParams &sp, bool scatter) {
  if (!scatter) return (size_t)sp.tp * sp.dp.limbs * sizeof(uint64_t) + (size_t)sp.S * sp.RA * sizeof(uint32_t);
  const size_t GR = (size_t)sort_a_groups(sp) * sp.RA;
  return (SORT_WARPS * GR + sp.RA) * sizeof(uint32_t);
}

// Signed digits of the pass-A tiles, written by the counting kernel and read
// by the scatter: dig[(tile * W + w) * tp + q] for point slot q.
GM_DEVI int64_t dig_index(int tile, int W, int w, int q, int tp) { return ((int64_t)tile * W + w) * tp + q; }

// Digits of the tile's points for windows [w0, w1), in (warp, round, lane)
// order: warp wp takes points [32 PPT wp, 32 PPT (wp + 1)), 32 per
// round; carry[] holds each point's carry into window w0 and is advanced.
// fn(w, q, d) for every window and point slot (d = 0: no entry).
template <int PPT, class Fn>
GM_DEVI void tile_digits(const uint64_t *sc, const TileA &ti, const SortParams &sp, int w0, int w1,
                         uint32_t (&carry)[PPT], Fn fn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, limbs = sp.dp.limbs;
  for (int w = w0; w < w1; w++) {
#pragma unroll
    for (int r = 0; r < PPT; r++) {
      const int q = warp * (32 * PPT) + r * 32 + lane;
      int d = 0;
      if (q < ti.np) d = signed_digit(sc + (size_t)q * limbs, limbs, w, sp.dp, carry[r]);
      fn(w, q, d);
      // counter updates of this round visible to every lane of the next
      __syncwarp();
    }
  }
}

// The tile's scalar words into shared memory with coalesced 128-bit loads
// from the first 16-byte boundary of the tile's rows (scalar rows are 8-byte
// aligned; with 5 limbs every other tile starts in the middle of a 16-byte
// pair); a leading and a trailing odd word take 64-bit loads.
GM_DEVI void stage_scalars(uint64_t *sc, const uint64_t *scalars, const TileA &ti, int limbs) {
  const uint64_t *src = scalars + ti.sc_row * limbs;
  const int64_t words = ti.np * limbs;
  if (words <= 0) return;
  const int head = (int)((reinterpret_cast<uintptr_t>(src) >> 3) & 1u);  // src is 8 mod 16
  const int64_t body = words - head;                                       // >= 0
  if (threadIdx.x == 0) {
    if (head) sc[0] = __ldg(src);
    if (body & 1) sc[words - 1] = __ldg(src + words - 1);
  }
  const uint4 *src4 = reinterpret_cast<const uint4 *>(src + head);
  for (int64_t k = threadIdx.x; k < (body >> 1); k += SA_THREADS) {
    const uint4 v = __ldg(src4 + k);
    sc[head + 2 * k] = (uint64_t)v.x | ((uint64_t)v.y << 32);
    sc[head + 2 * k + 1] = (uint64_t)v.z | ((uint64_t)v.w << 32);
  }
}

// Pass A, counting: the tile's signed digits (into dig) and its entries per
// (group in MSM, hi digit), counted with shared-memory atomics; writes every
// counter of the tile.
template <int PPT>
__global__ void __launch_bounds__(SA_THREADS) k_sort_a_count(const uint64_t *__restrict__ scalars, SortDesc sd,
                                                                  SortParams sp, uint32_t *__restrict__ cnt,
                                                                  int32_t *__restrict__ dig) {
  extern __shared__ uint64_t sort_smem[];
  const int limbs = sp.dp.limbs, RA = sp.RA, SR = sp.S * RA, W = sp.dp.W;
  uint64_t *sc = sort_smem;
  uint32_t *h = reinterpret_cast<uint32_t *>(sc + (size_t)sp.tp * limbs);  // [S][RA]
  const TileA ti = tile_a_info(sd, sp, blockIdx.x);
  stage_scalars(sc, scalars, ti, limbs);
  for (int k = threadIdx.x; k < SR; k += SA_THREADS) h[k] = 0;
  __syncthreads();
  const int shift = sp.passes == 2 ? sp.LB : 0;
  uint32_t carry[PPT] = {0};
  tile_digits<PPT>(sc, ti, sp, 0, W, carry, [&](int w, int q, int d) {
    dig[dig_index(blockIdx.x, W, w, q, sp.tp)] = d;
    if (d == 0) return;
    const uint32_t b = (uint32_t)(d < 0 ? -d : d) - 1u;
    atomicAdd(&h[(sp.S == 1 ? 0 : w) * RA + (b >> shift)], 1u);
  });
  __syncthreads();
  for (int k = threadIdx.x; k < SR; k += SA_THREADS) cnt[idx_a(ti, sp, k / RA, k % RA, ti.t)] = h[k];
}

// Pass A, scatter: cnt holds the scanned count matrix, dig the tile's
// digits.  Windows go in chunks of sort_a_chunk; per chunk: the per-warp
// counts of every (group, hi); their exclusive prefix over the warps on top
// of the tile's output range (and, with one group, of the earlier chunks'
// entries); then every entry at its warp's running position plus its rank
// among the warp's lanes.  Two passes: (key b, value) pairs into kv; one
// pass: values into entries (final order).  HB: bits of the hi digit; PPT:
// points per thread.
template <int HB, int PPT>
__global__ void __launch_bounds__(SA_THREADS) k_sort_a_scatter(const int32_t *__restrict__ dig, SortDesc sd,
                                                                    SortParams sp, const uint32_t *__restrict__ cnt,
                                                                    uint2 *__restrict__ kv,
                                                                    uint32_t *__restrict__ entries) {
  extern __shared__ uint32_t sa_smem[];
  const int RA = sp.RA, W = sp.dp.W;
  const int WC = sort_a_chunk(sp);
  const int GR = sort_a_groups(sp) * RA;
  uint32_t *wc = sa_smem;                 // [SORT_WARPS][GR]
  uint32_t *run = wc + SORT_WARPS * GR;   // [RA] earlier chunks (one group)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t *my = wc + warp * GR;
  // one block per (tile, chunk) with one group per window; one block per
  // tile (all chunks, in order) with the single group of table mode
  const int nch = sort_a_blocks_per_tile(sp);
  const int tile = blockIdx.x / nch;
  const int wbeg = sp.S == 1 ? 0 : (blockIdx.x % nch) * WC;
  const int wend = sp.S == 1 ? W : min(W, wbeg + WC);
  const TileA ti = tile_a_info(sd, sp, tile);
  for (int k = threadIdx.x; k < RA; k += SA_THREADS) run[k] = 0;
  const int shift = sp.passes == 2 ? sp.LB : 0;
  for (int w0 = wbeg; w0 < wend; w0 += WC) {
    const int w1 = min(W, w0 + WC);
    for (int k = threadIdx.x; k < SORT_WARPS * GR; k += SA_THREADS) wc[k] = 0;
    __syncthreads();
    int dg[SA_CHUNK_W][PPT];
#pragma unroll
    for (int j = 0; j < SA_CHUNK_W; j++) {
      const int w = w0 + j;
#pragma unroll
      for (int r = 0; r < PPT; r++) {
        const int q = warp * (32 * PPT) + r * 32 + lane;
        dg[j][r] = (w < w1 && q < ti.np) ? __ldg(dig + dig_index(tile, W, w, q, sp.tp)) : 0;
        if (dg[j][r] != 0) {
          const int d = dg[j][r];
          const uint32_t b = (uint32_t)(d < 0 ? -d : d) - 1u;
          atomicAdd(&my[(sp.S == 1 ? 0 : j) * RA + (b >> shift)], 1u);
        }
      }
    }
    __syncthreads();
    // running position of every (warp, group, hi) of the chunk: the tile's
    // range start plus the entries of the lower warps (and earlier chunks)
    const int GRc = (sp.S == 1 ? 1 : w1 - w0) * RA;
    for (int k = threadIdx.x; k < GRc; k += SA_THREADS) {
      const int g = k / RA, d = k % RA;
      const uint32_t base = cnt[idx_a(ti, sp, sp.S == 1 ? 0 : w0 + g, d, ti.t)];
      uint32_t acc = base + (sp.S == 1 ? run[d] : 0u);
      for (int j = 0; j < SORT_WARPS; j++) {
        const uint32_t x = wc[j * GR + k];
        wc[j * GR + k] = acc;
        acc += x;
      }
      if (sp.S == 1) run[d] = acc - base;
    }
    __syncthreads();
    const uint32_t rbase = (uint32_t)ti.base_off;
#pragma unroll
    for (int j = 0; j < SA_CHUNK_W; j++) {
      const int w = w0 + j;
      if (w >= w1) break;
      const uint32_t wofs = sd.pc_stride ? (uint32_t)((int64_t)w * sd.pc_stride) : 0u;
#pragma unroll
      for (int r = 0; r < PPT; r++) {
        const int q = warp * (32 * PPT) + r * 32 + lane;
        const int d = dg[j][r];
        const uint32_t b = (uint32_t)(d < 0 ? -d : d) - 1u;
        const uint32_t bin = d != 0 ? (b >> shift) : 0u;
        const uint32_t peers = same_bin_lanes<HB>(bin, d != 0);
        if (d != 0) {
          uint32_t *slot = &my[(sp.S == 1 ? 0 : j) * RA + bin];
          const uint32_t lower = peers & lanemask_lt();
          const uint32_t pos = *slot + __popc(lower);
          // record index < 2^31: 32-bit arithmetic
          const uint32_t rec = wofs + rbase + (uint32_t)q;
          const uint32_t val = (rec << 1) | (d < 0 ? 1u : 0u);
          if (sp.passes == 2)
            kv[pos] = make_uint2(b, val);
          else
            entries[pos] = val;
          __syncwarp(peers);
          if (lower == 0) *slot += __popc(peers);
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }
}

// Start of pass-A segment s (= group g, hi digit) in the pass-A output.
GM_DEVI uint32_t seg_start_of(const SortDesc &sd, const SortParams &sp, const uint32_t *posA, int64_t s) {
  if (s >= sp.NS) return __ldg(posA + sp.lenA);
  const int64_t g = s / sp.RA;
  const int hi = (int)(s % sp.RA);
  const int i = (int)(g / sp.S), s_local = (int)(g % sp.S);
  int64_t cbase, tiles;
  if (sd.point_start == nullptr) {
    cbase = 0;
    tiles = sp.tilesA;
  } else {
    const int f0 = __ldg(sd.tile_first + i);
    cbase = (int64_t)sp.S * sp.RA * f0;
    tiles = __ldg(sd.tile_first + i + 1) - f0;
  }
  return __ldg(posA + cbase + ((int64_t)s_local * sp.RA + hi) * tiles);
}

// Pass-B segments: seg[s] = start, tb[s] = tiles of segment s (scanned next).
static __global__ void k_sort_segments(SortDesc sd, SortParams sp, const uint32_t *__restrict__ posA,
                                       uint32_t *__restrict__ seg, uint32_t *__restrict__ tb) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s > sp.NS) return;
  const uint32_t a = seg_start_of(sd, sp, posA, s);
  seg[s] = a;
  if (s == sp.NS) return;
  const uint32_t e = seg_start_of(sd, sp, posA, s + 1);
  tb[s] = (e - a + SB_TILE - 1) / SB_TILE;
}

inline size_t sort_b_smem(const SortParams &sp, bool scatter) {
  if (!scatter) return (size_t)sp.RB * sizeof(uint32_t);
  return (size_t)(SORT_WARPS + 2) * sp.RB * sizeof(uint32_t) + 2 * (size_t)SB_TILE * sizeof(uint32_t);
}

struct TileB {
  int64_t s;
  int t, tiles;
  uint32_t e0, cb;
  int ne;
};

// Pass-B tile `tile` of the scanned tile counts tb (tb[NS] = total); false
// past the last tile.  Empty segments share tb values: the tile belongs to
// the last segment whose first tile is at or below it.
GM_DEVI bool tile_b_info(const SortParams &sp, const uint32_t *seg, const uint32_t *tb, int tile, TileB &tbi) {
  const int64_t NS = sp.NS;
  if (tile >= (int64_t)__ldg(tb + NS)) return false;
  int64_t lo = 0, hi = NS;  // tb[lo] <= tile < tb[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(tb + mid) <= (uint32_t)tile)
      lo = mid;
    else
      hi = mid;
  }
  const uint32_t tb0 = __ldg(tb + lo);
  tbi.s = lo;
  tbi.t = tile - (int)tb0;
  tbi.tiles = (int)(__ldg(tb + lo + 1) - tb0);
  tbi.cb = tb0;
  tbi.e0 = __ldg(seg + lo) + (uint32_t)tbi.t * SB_TILE;
  tbi.ne = (int)(min(__ldg(seg + lo + 1), tbi.e0 + (uint32_t)SB_TILE) - tbi.e0);
  return true;
}

// Pass B, counting: per-tile lo counts into cnt[RB tb[s] + lo tiles_s + t].
static __global__ void __launch_bounds__(SB_THREADS) k_sort_b_count(const uint2 *__restrict__ kv, SortParams sp,
                                                           const uint32_t *__restrict__ seg,
                                                           const uint32_t *__restrict__ tb, uint32_t *__restrict__ cnt) {
  extern __shared__ uint32_t sb_smem[];
  TileB tbi;
  if (!tile_b_info(sp, seg, tb, blockIdx.x, tbi)) return;
  const int RB = sp.RB;
  uint32_t *h = sb_smem;
  for (int k = threadIdx.x; k < RB; k += SB_THREADS) h[k] = 0;
  __syncthreads();
  for (int q = threadIdx.x; q < tbi.ne; q += SB_THREADS) atomicAdd(&h[__ldg(&kv[tbi.e0 + q].x) & (RB - 1)], 1u);
  __syncthreads();
  const int64_t cb = (int64_t)RB * tbi.cb;
  for (int d = threadIdx.x; d < RB; d += SB_THREADS) cnt[cb + (int64_t)d * tbi.tiles + tbi.t] = h[d];
}

// Pass B, scatter: cnt holds the scanned counts.  The tile's entries are
// ranked by lo (per-warp counts, their prefix over warps, lane ranks by
// ballots) into a shared-memory copy ordered by lo, which is then written
// out as contiguous runs.
template <int LB>
__global__ void __launch_bounds__(SB_THREADS) k_sort_b_scatter(const uint2 *__restrict__ kv, SortParams sp,
                                                             const uint32_t *__restrict__ seg,
                                                             const uint32_t *__restrict__ tb,
                                                             const uint32_t *__restrict__ cnt,
                                                             uint32_t *__restrict__ out) {
  extern __shared__ uint32_t sb_smem[];
  TileB tbi;
  if (!tile_b_info(sp, seg, tb, blockIdx.x, tbi)) return;
  const int RB = sp.RB;
  uint32_t *wc = sb_smem;                      // [SORT_WARPS][RB]
  uint32_t *tstart = wc + SORT_WARPS * RB;     // [RB] tile-local start of each lo
  uint32_t *gpos = tstart + RB;                // [RB] output start of (tile, lo)
  uint32_t *st_val = gpos + RB;                // [SB_TILE]
  uint32_t *st_bin = st_val + SB_TILE;         // [SB_TILE]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int k = tid; k < SORT_WARPS * RB; k += SB_THREADS) wc[k] = 0;
  __syncthreads();
  uint32_t *my = wc + warp * RB;
  uint32_t bin[SB_IPT];
#pragma unroll
  for (int r = 0; r < SB_IPT; r++) {
    const int q = warp * (32 * SB_IPT) + r * 32 + lane;
    bin[r] = q < tbi.ne ? (__ldg(&kv[tbi.e0 + q].x) & (uint32_t)(RB - 1)) : 0xffffffffu;
    if (bin[r] != 0xffffffffu) atomicAdd(&my[bin[r]], 1u);
  }
  __syncthreads();
  // tile-local start of every lo (exclusive scan over bins of the warp
  // totals), then each warp's start inside it
  {
    const int per = (RB + SB_THREADS - 1) / SB_THREADS;
    uint32_t sum = 0;
    for (int j = 0; j < per; j++) {
      const int d = tid * per + j;
      if (d < RB)
        for (int k = 0; k < SORT_WARPS; k++) sum += wc[k * RB + d];
    }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(sum, total);
    const int64_t cb = (int64_t)RB * tbi.cb;
    for (int j = 0; j < per; j++) {
      const int d = tid * per + j;
      if (d < RB) {
        tstart[d] = ex;
        gpos[d] = cnt[cb + (int64_t)d * tbi.tiles + tbi.t];
        for (int k = 0; k < SORT_WARPS; k++) {
          const uint32_t x = wc[k * RB + d];
          wc[k * RB + d] = ex;
          ex += x;
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < SB_IPT; r++) {
    const bool valid = bin[r] != 0xffffffffu;
    const uint32_t peers = same_bin_lanes<LB>(valid ? bin[r] : 0u, valid);
    if (valid) {
      const int q = warp * (32 * SB_IPT) + r * 32 + lane;
      const uint32_t lower = peers & lanemask_lt();
      const uint32_t local = my[bin[r]] + __popc(lower);
      st_val[local] = __ldg(&kv[tbi.e0 + q].y);
      st_bin[local] = bin[r];
      __syncwarp(peers);
      if (lower == 0) my[bin[r]] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  for (int k = tid; k < tbi.ne; k += SB_THREADS) {
    const uint32_t d = st_bin[k];
    out[gpos[d] + (uint32_t)k - tstart[d]] = st_val[k];
  }
}

// Bucket offsets from the scanned count matrices: offsets[k] for every key
// k = g*B + b, offsets[K] = number of entries.
static __global__ void k_sort_offsets(SortDesc sd, SortParams sp, int64_t K, const uint32_t *__restrict__ posA,
                                      const uint32_t *__restrict__ seg, const uint32_t *__restrict__ tb,
                                      const uint32_t *__restrict__ posB, uint32_t *__restrict__ offsets) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k > K) return;
  if (k == K) {
    offsets[K] = __ldg(posA + sp.lenA);
    return;
  }
  if (sp.passes == 1) {
    // key = g*B + b, b is the pass-A digit
    offsets[k] = seg_start_of(sd, sp, posA, k);
    return;
  }
  const int64_t s = k >> sp.LB;
  const uint32_t lo = (uint32_t)(k & (sp.RB - 1));
  const uint32_t t0 = __ldg(tb + s), tiles = __ldg(tb + s + 1) - t0;
  offsets[k] = tiles ? __ldg(posB + (int64_t)sp.RB * t0 + (int64_t)lo * tiles) : __ldg(seg + s);
}

// ---------------------------------------------------------------------------
// host side: digit split, workspace and launch sequence
// ---------------------------------------------------------------------------
struct SortLayout {
  SortParams sp;
  int64_t G = 0, maxM = 0;
  size_t o_cntA = 0, o_bsA = 0, o_dig = 0, o_kv = 0, o_seg = 0, o_tb = 0, o_bsT = 0, o_cntB = 0, o_bsB = 0;

  static int64_t scan_blocks(int64_t len) { return std::max<int64_t>(1, (len + SCAN_TILE - 1) / SCAN_TILE); }

  // count MSMs with P points in all, tilesA pass-A tiles (ceil(size_i / tp)
  // summed over the MSMs, tp = SA_THREADS * ppt); tabled: fixed-base window
  // table mode.
  template <class Carver>
  void plan(const DigitParams &dp, int count, int64_t P, int64_t tilesA, bool tabled, Carver &cv, int ppt = SA_PPT) {
    sp.dp = dp;
    sp.ppt = ppt;
    sp.tp = SA_THREADS * ppt;
    sp.S = tabled ? 1 : dp.W;
    const int nb = dp.c - 1;  // bits of a bucket index
    if (nb <= 8) {
      sp.passes = 1;
      sp.HB = nb;
      sp.LB = 0;
    } else {
      // at most 8 bits in pass A (its counters grow with 2^HB per tile)
      sp.passes = 2;
      sp.HB = std::min(8, nb / 2);
      sp.LB = nb - sp.HB;
    }
    sp.RA = 1 << sp.HB;
    sp.RB = 1 << sp.LB;
    G = (int64_t)count * sp.S;
    sp.NS = G * sp.RA;
    sp.tilesA = tilesA;
    sp.lenA = (int64_t)sp.S * sp.RA * tilesA;
    maxM = P * dp.W;
    o_cntA = cv.template take<uint32_t>((size_t)sp.lenA + 1);
    o_dig = cv.template take<int32_t>((size_t)tilesA * dp.W * sp.tp);
    o_bsA = cv.template take<uint32_t>((size_t)scan_blocks(sp.lenA));
    if (sp.passes == 2) {
      sp.tilesB_max = sp.NS + (maxM + SB_TILE - 1) / SB_TILE;
      sp.lenB = (int64_t)sp.RB * sp.tilesB_max;
      o_kv = cv.template take<uint2>((size_t)std::max<int64_t>(1, maxM));
      o_seg = cv.template take<uint32_t>((size_t)sp.NS + 1);
      o_tb = cv.template take<uint32_t>((size_t)sp.NS + 1);
      o_bsT = cv.template take<uint32_t>((size_t)scan_blocks(sp.NS));
      o_cntB = cv.template take<uint32_t>((size_t)sp.lenB + 1);
      o_bsB = cv.template take<uint32_t>((size_t)scan_blocks(sp.lenB));
    }
  }
};

// In-place exclusive scan of a[0, len); a[len] receives the total.
inline void scan_inplace(cudaStream_t s, uint32_t *a, int64_t len, uint32_t *bsum, int *launches) {
  const int64_t nb = SortLayout::scan_blocks(len);
  k_scan_blocksum<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(a, len, bsum);
  k_scan_top<<<1, SCAN_THREADS, 0, s>>>(bsum, (int)nb);
  k_scan_final<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(a, len, bsum, a);
  *launches += 3;
}

// Raises the opt-in shared-memory size of kernel fn on the current device
// when a launch needs more than 48 KB and more than the largest size set so
// far (slot: one per kernel instantiation).
inline cudaError_t smem_opt_in(const void *fn, int slot, size_t bytes) {
  static std::mutex mu;
  static int set[64][32] = {{0}};
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)bytes <= set[dev][slot]) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) set[dev][slot] = (int)bytes;
  return e;
}

template <int HB, int PPT>
cudaError_t launch_sort_a_scatter(cudaStream_t s, const SortParams &sp, const int32_t *dig, const SortDesc &sd,
                                  const uint32_t *cntA, uint2 *kv, uint32_t *entries) {
  const size_t sm = sort_a_smem(sp, true);
  cudaError_t e = smem_opt_in((const void *)k_sort_a_scatter<HB, PPT>, HB, sm);
  if (e != cudaSuccess) return e;
  k_sort_a_scatter<HB, PPT><<<(unsigned)(sp.tilesA * sort_a_blocks_per_tile(sp)), SA_THREADS, sm, s>>>(
      dig, sd, sp, cntA, kv, entries);
  return cudaSuccess;
}

template <int PPT>
cudaError_t launch_sort_a_scatter_hb(cudaStream_t s, const SortParams &sp, const int32_t *dig, const SortDesc &sd,
                                     const uint32_t *cntA, uint2 *kv, uint32_t *entries) {
  switch (sp.HB) {
    case 1: return launch_sort_a_scatter<1, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 2: return launch_sort_a_scatter<2, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 3: return launch_sort_a_scatter<3, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 4: return launch_sort_a_scatter<4, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 5: return launch_sort_a_scatter<5, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 6: return launch_sort_a_scatter<6, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 7: return launch_sort_a_scatter<7, PPT>(s, sp, dig, sd, cntA, kv, entries);
    case 8: return launch_sort_a_scatter<8, PPT>(s, sp, dig, sd, cntA, kv, entries);
    default: return cudaErrorInvalidValue;
  }
}

template <int PPT>
cudaError_t launch_sort_a_count(cudaStream_t s, const SortParams &sp, const uint64_t *scalars, const SortDesc &sd,
                                uint32_t *cntA, int32_t *dig) {
  const size_t sm = sort_a_smem(sp, false);
  cudaError_t e = smem_opt_in((const void *)k_sort_a_count<PPT>, 28 + PPT / 4, sm);
  if (e != cudaSuccess) return e;
  k_sort_a_count<PPT><<<(unsigned)sp.tilesA, SA_THREADS, sm, s>>>(scalars, sd, sp, cntA, dig);
  return cudaSuccess;
}

template <int LB>
cudaError_t launch_sort_b_scatter(cudaStream_t s, const SortParams &sp, const uint2 *kv, const uint32_t *seg,
                                  const uint32_t *tb, const uint32_t *cntB, uint32_t *entries) {
  const size_t sm = sort_b_smem(sp, true);
  cudaError_t e = smem_opt_in((const void *)k_sort_b_scatter<LB>, 16 + LB, sm);
  if (e != cudaSuccess) return e;
  k_sort_b_scatter<LB><<<(unsigned)sp.tilesB_max, SB_THREADS, sm, s>>>(kv, sp, seg, tb, cntB, entries);
  return cudaSuccess;
}

// The pass-A kernels for the tile sizes of SortLayout::plan (2, 4 or 8
// points per thread) and the digit widths HB in 1..8; the pass-B scatter for
// LB in 5..11.
inline cudaError_t sort_a_count(cudaStream_t s, const SortParams &sp, const uint64_t *scalars, const SortDesc &sd,
                                uint32_t *cntA, int32_t *dig) {
  switch (sp.ppt) {
    case 2: return launch_sort_a_count<2>(s, sp, scalars, sd, cntA, dig);
    case 4: return launch_sort_a_count<4>(s, sp, scalars, sd, cntA, dig);
    case 8: return launch_sort_a_count<8>(s, sp, scalars, sd, cntA, dig);
    default: return cudaErrorInvalidValue;
  }
}
inline cudaError_t sort_a_scatter(cudaStream_t s, const SortParams &sp, const int32_t *dig, const SortDesc &sd,
                                  const uint32_t *cntA, uint2 *kv, uint32_t *entries) {
  switch (sp.ppt) {
    case 2: return launch_sort_a_scatter_hb<2>(s, sp, dig, sd, cntA, kv, entries);
    case 4: return launch_sort_a_scatter_hb<4>(s, sp, dig, sd, cntA, kv, entries);
    case 8: return launch_sort_a_scatter_hb<8>(s, sp, dig, sd, cntA, kv, entries);
    default: return cudaErrorInvalidValue;
  }
}
inline cudaError_t sort_b_scatter(cudaStream_t s, const SortParams &sp, const uint2 *kv, const uint32_t *seg,
                                  const uint32_t *tb, const uint32_t *cntB, uint32_t *entries) {
  switch (sp.LB) {
    case 5: return launch_sort_b_scatter<5>(s, sp, kv, seg, tb, cntB, entries);
    case 6: return launch_sort_b_scatter<6>(s, sp, kv, seg, tb, cntB, entries);
    case 7: return launch_sort_b_scatter<7>(s, sp, kv, seg, tb, cntB, entries);
    case 8: return launch_sort_b_scatter<8>(s, sp, kv, seg, tb, cntB, entries);
    case 9: return launch_sort_b_scatter<9>(s, sp, kv, seg, tb, cntB, entries);
    case 10: return launch_sort_b_scatter<10>(s, sp, kv, seg, tb, cntB, entries);
    case 11: return launch_sort_b_scatter<11>(s, sp, kv, seg, tb, cntB, entries);
    default: return cudaErrorInvalidValue;
  }
}

// Enqueues the sort: entries[0, M) grouped by bucket key in point order and
// offsets[0, K] (K = G * B keys; offsets[K] = M).  Reads only the scalars.
inline cudaError_t sort_launch(cudaStream_t s, const SortLayout &L, char *ws, const uint64_t *scalars,
                               const SortDesc &sd, int64_t K, uint32_t *offsets, uint32_t *entries, int *launches) {
  const SortParams &sp = L.sp;
  cudaError_t e = smem_opt_in((const void *)k_sort_b_count, 9, sort_b_smem(sp, false));
  if (e != cudaSuccess) return e;
  auto *cntA = (uint32_t *)(ws + L.o_cntA);
  auto *bsA = (uint32_t *)(ws + L.o_bsA);
  auto *dig = (int32_t *)(ws + L.o_dig);
  e = sort_a_count(s, sp, scalars, sd, cntA, dig);
  if (e != cudaSuccess) return e;
  scan_inplace(s, cntA, sp.lenA, bsA, launches);
  uint32_t *seg = nullptr, *tb = nullptr, *cntB = nullptr;
  if (sp.passes == 1) {
    e = sort_a_scatter(s, sp, dig, sd, cntA, nullptr, entries);
    if (e != cudaSuccess) return e;
    *launches += 2;
  } else {
    auto *kv = (uint2 *)(ws + L.o_kv);
    seg = (uint32_t *)(ws + L.o_seg);
    tb = (uint32_t *)(ws + L.o_tb);
    cntB = (uint32_t *)(ws + L.o_cntB);
    e = sort_a_scatter(s, sp, dig, sd, cntA, kv, nullptr);
    if (e != cudaSuccess) return e;
    k_sort_segments<<<(unsigned)((sp.NS + 1 + 255) / 256), 256, 0, s>>>(sd, sp, cntA, seg, tb);
    scan_inplace(s, tb, sp.NS, (uint32_t *)(ws + L.o_bsT), launches);
    e = cudaMemsetAsync(cntB, 0, (size_t)sp.lenB * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    k_sort_b_count<<<(unsigned)sp.tilesB_max, SB_THREADS, sort_b_smem(sp, false), s>>>(kv, sp, seg, tb, cntB);
    scan_inplace(s, cntB, sp.lenB, (uint32_t *)(ws + L.o_bsB), launches);
    e = sort_b_scatter(s, sp, kv, seg, tb, cntB, entries);
    if (e != cudaSuccess) return e;
    *launches += 5;
  }
  k_sort_offsets<<<(unsigned)((K + 1 + 255) / 256), 256, 0, s>>>(sd, sp, K, cntA, seg, tb, cntB, offsets);
  (*launches)++;
  return cudaGetLastError();
}

}  // namespace gm
