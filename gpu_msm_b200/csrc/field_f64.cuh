// Montgomery product on the FP64 pipe: the same function as
// mont_mul_raw<true> (field.cuh) -- canonical inputs and output in 14 x 32-bit
// limbs, R = 2^448 -- computed with double-precision FMAs instead of 32-bit
// IMADs, so that it runs on the FP64 pipe while IMAD.HI-bound integer code
// runs on the FMA pipe.
//
// Scheme (the exact-split method of Emmart, Zheng and Weems, "Faster Modular
// Exponentiation Using Double Precision Floating Point Arithmetic on the GPU",
// ARITH 2018):
//   - operands become 9 limbs of 52 bits held as doubles;
//   - one 52 x 52-bit partial product a*b = H*2^52 + L is split exactly by
//       h = fma_rz(a, b, 2^104)                  = 2^104 + H*2^52
//       l = fma_rz(a, b, (2^104 + 2^52) - h)     = 2^52 + L
//     (rounding toward zero makes h truncate; the second FMA is exact), so
//     the bit patterns of h and l are fixed constants plus H and L;
//   - those bit patterns are summed as 64-bit integers into 18 columns of
//     52 bits; each column later subtracts (number of terms) x constant once;
//   - Montgomery reduction interleaves with the product in operand-scanning
//     order: row i of a*b completes column i, then step i clears it.  Eight
//     steps use a 52-bit m = t * (-p^-1) mod 2^52 (one 64-bit integer
//     product), a last one a 32-bit m, which clears 8*52 + 32 = 448 bits.  A
//     step's carry is (t >> 52) + (t mod 2^52 != 0), because t + lo(m*p0) is
//     a multiple of 2^52, so lo(m*p0) itself is never formed.  (The
//     interleaved order keeps fewer columns live than forming all of a*b
//     first: G1 2^20 accumulation 11.10 ms against 11.24 ms.)
//   - the result is the columns from bit 448 up, shifted into 14 x 32-bit
//     limbs, below 2p, then one conditional subtraction of p.
// Column sums stay below 36 * 2^52 < 2^58, so no column overflows.
#pragma once
#include "field.cuh"

namespace gm {
namespace f64 {

constexpr uint64_t MASK52 = (1ull << 52) - 1;
constexpr uint64_t BITS_2_52 = 1075ull << 52;   // bit pattern of 2^52
constexpr uint64_t BITS_2_104 = 1127ull << 52;  // bit pattern of 2^104
constexpr uint64_t PINV52 = 0x3fd900035fffdull;  // -p^-1 mod 2^52

// p in 52-bit limbs (the constant of src/fp.cu:15 regrouped)
GM_HDI constexpr uint64_t p52(int j) {
  return j == 0   ? 0xc0026aab0aaabull
         : j == 1 ? 0x28c573b5cc311ull
         : j == 2 ? 0x23acdee56ee45ull
         : j == 3 ? 0x1602824e6dc3eull
         : j == 4 ? 0x20f75a64bbac7ull
         : j == 5 ? 0x95a4b78a02fe3ull
         : j == 6 ? 0x34965aad64000ull
         : j == 7 ? 0x28c5e535200fcull
                  : 0x3cdee0fbull;
}

// Offset terms in column k once all 81 operand products, the reduction steps
// s < nsteps (52-bit m; no low half for j = 0) and, with the last step, the
// 32-bit step have been added.
GM_HDI constexpr int lo_terms(int k, int nsteps, bool last) {
  int n = 0;
  for (int x = 0; x < 9; x++)
    for (int y = 0; y < 9; y++) n += (x + y == k);
  for (int s = 0; s < nsteps; s++)
    for (int j = 1; j < 9; j++) n += (s + j == k);
  if (last)
    for (int j = 1; j < 9; j++) n += (8 + j == k);
  return n;
}
GM_HDI constexpr int hi_terms(int k, int nsteps, bool last) {
  int n = 0;
  for (int x = 0; x < 9; x++)
    for (int y = 0; y < 9; y++) n += (x + y + 1 == k);
  for (int s = 0; s < nsteps; s++)
    for (int j = 0; j < 9; j++) n += (s + j + 1 == k);
  if (last)
    for (int j = 0; j < 9; j++) n += (8 + j + 1 == k);
  return n;
}
GM_HDI constexpr uint64_t offset(int k, int nsteps, bool last) {
  return (uint64_t)lo_terms(k, nsteps, last) * BITS_2_52 + (uint64_t)hi_terms(k, nsteps, last) * BITS_2_104;
}

GM_DEVI double as_d(uint64_t x) { return __longlong_as_double((long long)x); }
GM_DEVI uint64_t as_u(double d) { return (uint64_t)__double_as_longlong(d); }
// x < 2^52 -> the double x, exactly
GM_DEVI double to_d(uint64_t x) { return as_d(x | BITS_2_52) - 0x1p52; }

// bits [52 i, 52 i + 52) of the 448-bit value in 14 x 32-bit limbs
GM_DEVI uint64_t limb52(const uint32_t w[NL], int i) {
  const int bit = 52 * i;
  uint64_t v = 0;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int word = bit / 32 + q;
    const int sh = 32 * q - bit % 32;  // position of the word's bit 0 in v
    if (word < NL) {
      if (sh >= 0 && sh < 64)
        v |= (uint64_t)w[word] << sh;
      else if (sh < 0)
        v |= (uint64_t)w[word] >> (-sh);
    }
  }
  return v & MASK52;
}

// column lo += bits(2^52 + L), column hi += bits(2^104 + H) for a*b = H 2^52 + L
GM_DEVI void split_acc(double a, double b, uint64_t &lo, uint64_t &hi) {
  const double h = __fma_rz(a, b, 0x1p104);
  const double l = __fma_rz(a, b, (0x1p104 + 0x1p52) - h);
  lo += as_u(l);
  hi += as_u(h);
}

GM_DEVI void mont_mul(uint32_t r[NL], const uint32_t a[NL], const uint32_t b[NL]) {
  double bd[9];
#pragma unroll
  for (int i = 0; i < 9; i++) bd[i] = to_d(limb52(b, i));
  uint64_t col[18];
#pragma unroll
  for (int k = 0; k < 18; k++) col[k] = 0;
  // operand scanning: row i of a*b completes column i, then reduction step
  // i clears it (columns i+1 .. i+9 are the only live ones)
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const double ai = to_d(limb52(a, i));
#pragma unroll
    for (int j = 0; j < 9; j++) split_acc(ai, bd[j], col[i + j], col[i + j + 1]);
    const uint64_t t = col[i] - offset(i, i, false);  // exact value of column i
    const uint64_t tl = t & MASK52;
    const double m = to_d((tl * PINV52) & MASK52);
    col[i + 1] += (t >> 52) + (tl != 0 ? 1u : 0u);
    col[i + 1] += as_u(__fma_rz(m, (double)p52(0), 0x1p104));
#pragma unroll
    for (int j = 1; j < 9; j++) split_acc(m, (double)p52(j), col[i + j], col[i + j + 1]);
  }
  {
    const double a8 = to_d(limb52(a, 8));
#pragma unroll
    for (int j = 0; j < 9; j++) split_acc(a8, bd[j], col[8 + j], col[9 + j]);
  }
  // last step: a 32-bit m clears bits 416..447
  const uint64_t t8 = col[8] - offset(8, 8, false);
  const double m8 = to_d((uint32_t)t8 * (uint32_t)PINV52);
  uint64_t e8;
  {
    const double h = __fma_rz(m8, (double)p52(0), 0x1p104);
    const double l = __fma_rz(m8, (double)p52(0), (0x1p104 + 0x1p52) - h);
    e8 = t8 + (as_u(l) - BITS_2_52);
    col[9] += as_u(h);
  }
#pragma unroll
  for (int j = 1; j < 9; j++) split_acc(m8, (double)p52(j), col[8 + j], col[9 + j]);
  // columns 8..17 -> 52-bit limbs c of C; the result is C >> 32
  uint64_t c[10];
  uint64_t carry = e8 >> 52;
  c[0] = e8 & MASK52;
#pragma unroll
  for (int k = 9; k < 18; k++) {
    const uint64_t v = col[k] - offset(k, 8, true) + carry;
    c[k - 8] = v & MASK52;
    carry = v >> 52;
  }
#pragma unroll
  for (int w = 0; w < NL; w++) {
    const int bit = 32 + 32 * w;
    const int L = bit / 52, S = bit % 52;
    uint64_t v = c[L] >> S;
    if (L + 1 < 10) v |= c[L + 1] << (52 - S);
    r[w] = (uint32_t)v;
  }
  cond_sub<false>(r);
}

}  // namespace f64

// Out of line, like fp_mul_call: one copy of the product per kernel.
static __device__ __noinline__ fp_t fp_mul_f64_call(fp_t a, fp_t b) {
  fp_t r;
  f64::mont_mul(r.v, a.v, b.v);
  return r;
}
// The accumulation-loop policy with the FP64 product (squares through it too)
struct FpOutF64 : Fp {
  GM_DEVI static fp_t mul(const fp_t &a, const fp_t &b) { return fp_mul_f64_call(a, b); }
  GM_DEVI static fp_t sqr(const fp_t &a) { return fp_mul_f64_call(a, a); }
};

}  // namespace gm
