"""Seeded synthetic MSM workloads with the distributions of the benchmark
configurations: scalars uniform in [0, r) with 1% set to 0 and 1% set to 1,
and bases P_i = t_i * G with t_i uniform in [1, r) and 2% of the bases
duplicated from other entries (so bucket sums hit the doubling case).

The bases are produced on the device from their discrete logs t_i
(``generator_mul_batch``); because t_i is known, the exact MSM result is
(sum_i k_i t_i mod r) * G, which gives a full-size correctness check.

No public dataset is involved; seeds replace it.
"""
from __future__ import annotations

import numpy as np

# scalar-field order r = u^4 - u^2 + 1 for the BLS12 parameter
# u = -0x6008204000000020001 of this curve (p = (u-1)^2 r / 3 + u)
U_PARAM = -0x6008204000000020001
R_ORDER = U_PARAM ** 4 - U_PARAM ** 2 + 1
# base-field prime p = (u - 1)^2 r / 3 + u (446 bits)
P_MODULUS = (U_PARAM - 1) ** 2 * R_ORDER // 3 + U_PARAM
R_LIMBS = np.array([(R_ORDER >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(5)], dtype=np.uint64)
SCALAR_LIMBS = 5
SCALAR_BITS = R_ORDER.bit_length()  # 299


def _lt_r(s: np.ndarray) -> np.ndarray:
    """Row-wise s < r for (n, 5) little-endian limbs."""
    lt = np.zeros(len(s), dtype=bool)
    eq = np.ones(len(s), dtype=bool)
    for i in range(4, -1, -1):
        lt |= eq & (s[:, i] < R_LIMBS[i])
        eq &= s[:, i] == R_LIMBS[i]
    return lt


def uniform_below_r(rng: np.random.Generator, n: int) -> np.ndarray:
    """n scalars uniform in [0, r) as (n, 5) u64 limbs (rejection sampling)."""
    out = np.empty((n, 5), dtype=np.uint64)
    filled = 0
    top_mask = np.uint64((1 << (SCALAR_BITS - 256)) - 1)
    while filled < n:
        m = int((n - filled) * 1.7) + 16
        cand = rng.integers(0, 2 ** 64, size=(m, 5), dtype=np.uint64)
        cand[:, 4] &= top_mask
        ok = cand[_lt_r(cand)]
        take = min(len(ok), n - filled)
        out[filled:filled + take] = ok[:take]
        filled += take
    return out


def make_scalars(n: int, seed: int = 42, zero_frac: float = 0.01, one_frac: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = uniform_below_r(rng, n)
    idx = rng.permutation(n)
    nz, no = int(n * zero_frac), int(n * one_frac)
    s[idx[:nz]] = 0
    s[idx[nz:nz + no]] = 0
    s[idx[nz:nz + no], 0] = 1
    return s


def make_base_logs(n: int, seed: int = 4242, dup_frac: float = 0.02) -> np.ndarray:
    """Discrete logs t_i in [1, r) of the bases, with dup_frac duplicated."""
    rng = np.random.default_rng(seed)
    t = uniform_below_r(rng, n)
    zero = ~np.any(t != 0, axis=1)
    t[zero, 0] = 1
    nd = int(n * dup_frac)
    if nd and n > 1:
        dst = rng.choice(n, size=nd, replace=False)
        src = rng.integers(0, n, size=nd)
        t[dst] = t[src]
    return t


def limbs_to_ints(a: np.ndarray) -> list:
    a = np.asarray(a, dtype=np.uint64)
    cols = [[int(v) for v in a[:, i]] for i in range(a.shape[1])]
    return [sum(c[i] << (64 * i) for i in range(len(cols))) for c in zip(*cols)]


def expected_log(scalars: np.ndarray, logs: np.ndarray) -> int:
    """sum_i k_i t_i mod r: the discrete log of the exact MSM result."""
    ks = limbs_to_ints(scalars)
    ts = limbs_to_ints(logs)
    acc = 0
    for k, t in zip(ks, ts):
        acc += k * t
    return acc % R_ORDER


def limbs16(a: np.ndarray) -> np.ndarray:
    """(n, L) little-endian u64 limbs -> (n, 4L) float64 array of their
    16-bit limbs (each an exact integer below 2^16)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a.view(np.uint16).reshape(len(a), -1).astype(np.float64)


# rows per exact product chunk: n (2^16 - 1)^2 < 2^53 keeps every partial sum
# of the float64 matrix product an exact integer
_DOT_CHUNK = 1 << 20


def dot_log(k16: np.ndarray, t16: np.ndarray) -> int:
    """sum_i k_i t_i mod r from 16-bit limb rows (limbs16): the limb-product
    sums sum_i k_i[a] t_i[b] are computed exactly as float64 matrix products
    over chunks of at most 2^20 rows, then weighted by 2^(16 (a + b))."""
    n = len(k16)
    if n != len(t16):
        raise ValueError("scalars and logs must have the same number of rows")
    acc = 0
    for r0 in range(0, n, _DOT_CHUNK):
        m = (k16[r0:r0 + _DOT_CHUNK].T @ t16[r0:r0 + _DOT_CHUNK]).astype(np.int64)
        la, lb = m.shape
        for c in range(la + lb - 1):
            a0, a1 = max(0, c - lb + 1), min(la - 1, c)
            s = int(sum(int(m[a, c - a]) for a in range(a0, a1 + 1)))
            acc += s << (16 * c)
    return acc % R_ORDER


def expected_logs(sizes, scalars: np.ndarray, logs: np.ndarray, base_offsets=None) -> list:
    """Discrete logs of the exact results of consecutive MSMs: MSM j takes the
    next sizes[j] scalar rows and the logs [base_offsets[j], + sizes[j]) of
    the table (prefixes when base_offsets is None)."""
    k16 = limbs16(scalars)
    t16 = limbs16(logs)
    out, row = [], 0
    for j, s in enumerate(np.asarray(sizes, dtype=np.int64)):
        s = int(s)
        o = 0 if base_offsets is None else int(base_offsets[j])
        out.append(dot_log(k16[row:row + s], t16[o:o + s]))
        row += s
    return out


def int_to_limbs(v: int, n: int = 5) -> np.ndarray:
    return np.array([(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def mixed_sizes(count: int, lo_log2: float, hi_log2: float, seed: int = 7) -> np.ndarray:
    """Log-uniform integer sizes floor(2^U), U ~ Uniform[lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.floor(2.0 ** rng.uniform(lo_log2, hi_log2, size=count)).astype(np.int64)


def signed_digit_counts(scalars: np.ndarray, c: int) -> np.ndarray:
    """Number of non-zero signed c-bit digits per window (the entries the
    bucket accumulation processes), computed the way the digit kernel
    decomposes scalars: d = raw + carry; d > 2^(c-1) -> d - 2^c, carry 1."""
    s = np.asarray(scalars, dtype=np.uint64)
    if s.ndim == 1:
        s = s.reshape(-1, 1)
    limbs = s.shape[1]
    W = (64 * limbs) // c + 1
    B = 1 << (c - 1)
    carry = np.zeros(len(s), dtype=np.int64)
    counts = np.zeros(W, dtype=np.int64)
    mask = np.uint64((1 << c) - 1)
    for w in range(W):
        off = w * c
        l, sh = off // 64, off % 64
        if l >= limbs:
            raw = np.zeros(len(s), dtype=np.int64)
        else:
            v = s[:, l] >> np.uint64(sh)
            if sh + c > 64 and l + 1 < limbs:
                v = v | (s[:, l + 1] << np.uint64(64 - sh))
            raw = (v & mask).astype(np.int64)
        v = raw + carry
        neg = v > B
        d = np.where(neg, v - 2 * B, v)
        carry = neg.astype(np.int64)
        counts[w] = int(np.count_nonzero(d))
    return counts


def msm_roofline_imad(n: int, group: int = 1) -> float:
    """Algorithmic IMAD count of an MSM of n points, fixed independently of the
    implementation: 798 IMAD per Fp multiplication (CIOS over 14 x 32-bit
    limbs), k = 1 (G1) or 3 (G2) Fp multiplications per field multiplication,
    and min over c of [10 n W + 28 2^(c-1) W + 10 c W] field multiplications
    with W = ceil(300 / c) signed windows."""
    k = 1 if group == 1 else 3
    best = min(10 * n * (-(-300 // c)) + 28 * 2 ** (c - 1) * (-(-300 // c)) + 10 * c * (-(-300 // c))
               for c in range(4, 23))
    return 798.0 * k * best
