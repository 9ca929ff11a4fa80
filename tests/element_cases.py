"""Seeded cases for the single-element operations (the reference's stream
APIs fp_*_async / fp2_*_async / point_*_async and the host-pointer *_gpu
helpers) and their expected values from the pure-Python oracle.

Field values are plain ints; points are (x, y, infinity) triples whose
coordinates are stored as given (Montgomery form for the point operations,
like the reference's).  Shared by the oracle pin (CPU, against the
reference's own host code) and the GPU parity test.
"""
from __future__ import annotations

import random

import numpy as np

import oracle
from oracle import pyref

P = pyref.P
R = pyref.R_MONT % P
R_INV = pyref.R_INV


def fp_np(v: int) -> np.ndarray:
    return oracle.int_to_limbs(v, 7)


def fp2_np(v) -> np.ndarray:
    return np.concatenate([oracle.int_to_limbs(v[0], 7), oracle.int_to_limbs(v[1], 7)])


def fp_int(a) -> int:
    return oracle.limbs_to_int(np.asarray(a, dtype=np.uint64)[:7])


def fp2_int(a):
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    return (oracle.limbs_to_int(a[:7]), oracle.limbs_to_int(a[7:14]))


def _square(rnd):
    x = rnd.randrange(1, P)
    return x * x % P


def fp_cases(seed: int = 11):
    """(op, a, b, c, arg) tuples covering every Fp op and its edge values."""
    rnd = random.Random(seed)
    vals = [0, 1, 2, P - 1, (P - 1) // 2] + [rnd.randrange(P) for _ in range(4)]
    pairs = [(a, b) for a in vals[:5] for b in vals[:5]] + [(rnd.randrange(P), rnd.randrange(P)) for _ in range(6)]
    cases = []
    for a, b in pairs:
        for op in ("add", "sub", "mul", "div", "mont_mul", "cmp"):
            cases.append((op, a, b, 0, 0))
    for a in vals:
        for op in ("neg", "inv", "copy", "to_mont", "from_mont", "is_zero", "is_one", "is_qr", "sqrt"):
            cases.append((op, a, 0, 0, 0))
    for _ in range(4):
        q = _square(rnd)
        cases += [("sqrt", q, 0, 0, 0), ("is_qr", q, 0, 0, 0)]
    cases += [("sqrt", P - 1, 0, 0, 0), ("is_qr", P - 1, 0, 0, 0)]  # -1 is a non-residue (p = 3 mod 4)
    cases += [("zero", 0, 0, 0, 0), ("one", 0, 0, 0, 0)]
    a, c = rnd.randrange(P), rnd.randrange(P)
    cases += [("cmov", a, 0, c, 0), ("cmov", a, 0, c, 1), ("cmov", a, 0, c, 2), ("cmov", a, 0, c, 3)]
    for e in (0, 1, 2, 3, 65537, 2 ** 64 - 1, rnd.getrandbits(64)):
        cases += [("pow_u64", rnd.randrange(P), 0, 0, e), ("pow_u64", 0, 0, 0, e)]
    return cases


def fp2_cases(seed: int = 12):
    rnd = random.Random(seed)
    r = lambda: (rnd.randrange(P), rnd.randrange(P))  # noqa: E731
    vals = [(0, 0), (1, 0), (0, 1), (P - 1, P - 1), (P - 1, 0)] + [r() for _ in range(3)]
    pairs = [(a, b) for a in vals[:5] for b in vals[:5]] + [(r(), r()) for _ in range(6)]
    cases = []
    for a, b in pairs:
        for op in ("add", "sub", "mul", "div", "mont_mul", "cmp"):
            cases.append((op, a, b, (0, 0), 0))
    for a in vals:
        for op in ("square", "neg", "conjugate", "inv", "copy", "mul_by_i", "frobenius", "is_zero", "is_one"):
            cases.append((op, a, (0, 0), (0, 0), 0))
    a, c = r(), r()
    cases += [("cmov", a, (0, 0), c, 0), ("cmov", a, (0, 0), c, 1)]
    return cases


def _mont_pt(pt, group):
    x, y, inf = pt
    if group == 1:
        return (pyref.to_mont(x), pyref.to_mont(y), inf)
    return ((pyref.to_mont(x[0]), pyref.to_mont(x[1])), (pyref.to_mont(y[0]), pyref.to_mont(y[1])), inf)


def _std_pt(pt, group):
    x, y, inf = pt
    if group == 1:
        return (pyref.from_mont(x), pyref.from_mont(y), inf)
    return ((pyref.from_mont(x[0]), pyref.from_mont(x[1])), (pyref.from_mont(y[0]), pyref.from_mont(y[1])), inf)


def point_cases(group: int, seed: int = 13, heavy: bool = True):
    """(op, p, q, scalar, limbs) with p, q Montgomery-form triples; scalar is
    an int (limbs 0 -> the u64 entry point)."""
    rnd = random.Random(seed + group)
    gen = pyref.g1() if group == 1 else pyref.g2()
    zero = 0 if group == 1 else (0, 0)

    def mult(k):
        v = pyref.mul(gen, k, group)
        return (zero, zero, True) if v is None else (v[0], v[1], False)

    Pp, Q = mult(rnd.randrange(1, pyref.R_ORDER)), mult(rnd.randrange(1, pyref.R_ORDER))
    F = pyref._field(group)
    negP = (Pp[0], F.neg(Pp[1]), False)
    inf = (zero, zero, True)
    junk_inf = (Q[0], Q[1], True)  # infinity flag with coordinates left in place
    pts = [Pp, Q, negP, inf]
    cases = []
    for a in pts:
        for b in pts + [junk_inf]:
            cases.append(("add", a, b, 0, 0))
    cases.append(("add", Pp, Pp, 0, 0))
    cases.append(("add", junk_inf, Q, 0, 0))
    # same x, unrelated y (not on the curve): the reference's lambda = 0 branch
    cases.append(("add", Pp, (Pp[0], F.add(Pp[1], F.small(5)), False), 0, 0))
    for a in pts + [junk_inf]:
        for op in ("double", "neg", "to_mont", "from_mont"):
            cases.append((op, a, None, 0, 0))
    if group == 1:
        t2 = (P - 1, 0, False)  # (-1, 0): the 2-torsion point of y^2 = x^3 + 1
        cases += [("double", t2, None, 0, 0), ("add", t2, t2, 0, 0), ("scalar_mul_u64", t2, None, 3, 0)]
    cases.append(("at_infinity", None, None, 0, 0))
    for k in (0, 1, 2, 3, rnd.getrandbits(64), 2 ** 64 - 1):
        cases.append(("scalar_mul_u64", Pp, None, k, 0))
    cases.append(("scalar_mul_u64", inf, None, 7, 0))
    if heavy:
        for k in (0, 1, pyref.R_ORDER - 1, pyref.R_ORDER, rnd.randrange(pyref.R_ORDER)):
            cases.append(("scalar_mul", Pp, None, k, 5))
        cases.append(("scalar_mul", Pp, None, rnd.getrandbits(100), 2))
        cases.append(("scalar_mul", Pp, None, 5, 0))  # no limbs: a zero scalar
    return [(op, _mont_pt(a, group) if a is not None else None, _mont_pt(b, group) if b is not None else None, k,
             limbs) for op, a, b, k, limbs in cases]


def expected_point(op, p, q, k, limbs, group):
    """Expected Montgomery-form triple for one case of point_cases."""
    zero = 0 if group == 1 else (0, 0)
    if op in ("to_mont", "from_mont"):
        if p[2]:
            return (zero, zero, True)
        f = (lambda v: v * R % P) if op == "to_mont" else (lambda v: v * R_INV % P)
        if group == 1:
            return (f(p[0]), f(p[1]), False)
        return ((f(p[0][0]), f(p[0][1])), (f(p[1][0]), f(p[1][1])), False)
    if op == "scalar_mul" and limbs == 0:
        k = 0
    sp = _std_pt(p, group) if p is not None else None
    sq = _std_pt(q, group) if q is not None else None
    r = pyref.point_elem(op, sp, sq, k, group)
    return _mont_pt(r, group)


def point_np(pt, group):
    dt = oracle.G1 if group == 1 else oracle.G2
    a = np.zeros(1, dtype=dt)
    if pt is None:
        return a
    x, y, inf = pt
    if group == 1:
        a["x"][0], a["y"][0] = fp_np(x), fp_np(y)
    else:
        a["x"][0] = fp2_np(x).reshape(2, 7)
        a["y"][0] = fp2_np(y).reshape(2, 7)
    a["infinity"][0] = 1 if inf else 0
    return a


def point_from_np(a, group):
    a = a.reshape(-1)[0]
    if group == 1:
        return (fp_int(a["x"]), fp_int(a["y"]), bool(a["infinity"]))
    return (fp2_int(a["x"]), fp2_int(a["y"]), bool(a["infinity"]))
