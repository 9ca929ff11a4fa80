"""CPU oracle for the BLS12-446 MSM path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
library (``gpu_msm_b200``) never imports it.

Three independent restatements of the reference (pdroalves/gpu_msm) live here:

* ``liboracle.so`` -- plain C (``oracle.c``) restating src/fp.cu, src/fp2.cu
  and src/curve.cu, with a reference-structured Pippenger and a naive
  double-and-add MSM;
* ``_ref/libref.so`` -- the reference's own host code compiled from its
  sources (``ref_shim.cu``), present when the reference tree was available at
  build time;
* ``pyref`` -- pure-Python big-integer arithmetic for small cases.

Parity pin: ``tests/test_oracle.py`` checks all three against each other and
against the known-answer vectors of the reference's tests
(``tests/golden/``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import pyref

_HERE = os.path.dirname(os.path.abspath(__file__))

# numpy dtypes byte-compatible with the reference structs (include/fp.h:13,
# include/fp2.h:10, include/curve.h:13-43): 56, 112, 120, 232, 168 and 336 bytes.
FP = np.dtype(("<u8", (7,)))
FP2 = np.dtype(("<u8", (2, 7)))
G1 = np.dtype([("x", "<u8", (7,)), ("y", "<u8", (7,)), ("infinity", "u1"), ("_pad", "u1", (7,))])
G2 = np.dtype([("x", "<u8", (2, 7)), ("y", "<u8", (2, 7)), ("infinity", "u1"), ("_pad", "u1", (7,))])
G1P = np.dtype([("X", "<u8", (7,)), ("Y", "<u8", (7,)), ("Z", "<u8", (7,))])
G2P = np.dtype([("X", "<u8", (2, 7)), ("Y", "<u8", (2, 7)), ("Z", "<u8", (2, 7))])
assert G1.itemsize == 120 and G2.itemsize == 232 and G1P.itemsize == 168 and G2P.itemsize == 336

P = pyref.P
R_ORDER = pyref.R_ORDER

_lib = None
_ref = None


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def lib():
    """The C restatement (built by ``oracle/Makefile``)."""
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        _lib = ctypes.CDLL(path)
    return _lib


def ref_lib():
    """The reference's own host code, or None when it was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libref.so")
        if not os.path.exists(path):
            return None
        _ref = ctypes.CDLL(path)
    return _ref


# ---------------------------------------------------------------------------
# int <-> limb helpers
# ---------------------------------------------------------------------------

def int_to_limbs(v: int, n: int = 7) -> np.ndarray:
    return np.array([(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def limbs_to_int(a) -> int:
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    return sum(int(x) << (64 * i) for i, x in enumerate(a))


def ints_to_fp_array(vals) -> np.ndarray:
    out = np.zeros((len(vals), 7), dtype=np.uint64)
    for i, v in enumerate(vals):
        out[i] = int_to_limbs(v)
    return out


def fp_array_to_ints(arr) -> list:
    arr = np.asarray(arr, dtype=np.uint64).reshape(-1, 7)
    return [limbs_to_int(r) for r in arr]


# ---------------------------------------------------------------------------
# batched field ops through the C restatement
# ---------------------------------------------------------------------------

def _binop(name, a, b, dt):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros_like(a)
    n = a.size // (7 if dt is FP else 14)
    getattr(lib(), name)(_ptr(out), _ptr(a), _ptr(b), ctypes.c_int64(n))
    return out


def fp_mont_mul(a, b):
    return _binop("orc_fp_mont_mul_batch", a, b, FP)


def fp_mul(a, b):
    return _binop("orc_fp_mul_batch", a, b, FP)


def fp2_mont_mul(a, b):
    return _binop("orc_fp2_mont_mul_batch", a, b, FP2)


def fp2_mul(a, b):
    return _binop("orc_fp2_mul_batch", a, b, FP2)


def fp_to_mont(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().orc_fp_to_mont_batch(_ptr(out), _ptr(a), ctypes.c_int64(a.size // 7))
    return out


def fp_from_mont(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    out = np.zeros_like(a)
    lib().orc_fp_from_mont_batch(_ptr(out), _ptr(a), ctypes.c_int64(a.size // 7))
    return out


# ---------------------------------------------------------------------------
# points
# ---------------------------------------------------------------------------

def g1_generator(mont: bool = True) -> np.ndarray:
    g = np.zeros(1, dtype=G1)
    lib().orc_g1_generator(_ptr(g))
    if mont:
        lib().orc_g1_to_mont(_ptr(g), _ptr(g))
    return g


def g2_generator(mont: bool = True) -> np.ndarray:
    g = np.zeros(1, dtype=G2)
    lib().orc_g2_generator(_ptr(g))
    if mont:
        lib().orc_g2_to_mont(_ptr(g), _ptr(g))
    return g


def _grp(group):
    return (G1, "g1") if group == 1 else (G2, "g2")


def to_mont(points, group=1):
    dt, g = _grp(group)
    pts = np.ascontiguousarray(points, dtype=dt)
    out = np.zeros_like(pts)
    fn = getattr(lib(), f"orc_{g}_to_mont")
    for i in range(len(pts)):
        fn(ctypes.c_void_p(out.ctypes.data + i * dt.itemsize), ctypes.c_void_p(pts.ctypes.data + i * dt.itemsize))
    return out


def from_mont(points, group=1):
    dt, g = _grp(group)
    pts = np.ascontiguousarray(points, dtype=dt)
    out = np.zeros_like(pts)
    fn = getattr(lib(), f"orc_{g}_from_mont")
    for i in range(len(pts)):
        fn(ctypes.c_void_p(out.ctypes.data + i * dt.itemsize), ctypes.c_void_p(pts.ctypes.data + i * dt.itemsize))
    return out


def scalar_mul(point, k: int, group=1, fast=True, limbs=5):
    """k * P for one Montgomery-form affine point (k < 2^(64*limbs))."""
    dt, g = _grp(group)
    p = np.ascontiguousarray(point, dtype=dt).reshape(1)
    out = np.zeros(1, dtype=dt)
    ks = int_to_limbs(k, limbs)
    fn = getattr(lib(), f"orc_{g}_scalar_mul_fast" if fast else f"orc_{g}_scalar_mul")
    fn(_ptr(out), _ptr(p), _ptr(ks), ctypes.c_int(limbs))
    return out


def msm_pippenger(points, scalars, group=1, threads=None):
    """Reference-structured CPU Pippenger; canonical affine (Montgomery)."""
    dt, g = _grp(group)
    pts = np.ascontiguousarray(points, dtype=dt)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    n = len(pts)
    limbs = sc.size // max(n, 1) if n else 1
    out = np.zeros(1, dtype=dt)
    threads = threads or os.cpu_count() or 1
    getattr(lib(), f"orc_{g}_msm_pippenger")(_ptr(out), _ptr(pts), _ptr(sc), ctypes.c_int(limbs),
                                             ctypes.c_int64(n), ctypes.c_int(threads))
    return out


def msm_naive(points, scalars, group=1, threads=None):
    """Naive double-and-add MSM; canonical affine (Montgomery)."""
    dt, g = _grp(group)
    pts = np.ascontiguousarray(points, dtype=dt)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    n = len(pts)
    limbs = sc.size // max(n, 1) if n else 1
    out = np.zeros(1, dtype=dt)
    threads = threads or os.cpu_count() or 1
    getattr(lib(), f"orc_{g}_msm_naive")(_ptr(out), _ptr(pts), _ptr(sc), ctypes.c_int(limbs),
                                         ctypes.c_int64(n), ctypes.c_int(threads))
    return out


def ref_msm_pippenger(points, scalars, group=1, threads=None):
    """The reference's own host functions arranged as its MSM driver does.
    Returns (affine Montgomery, projective Montgomery) or None if unbuilt."""
    r = ref_lib()
    if r is None:
        return None
    dt, g = _grp(group)
    pdt = G1P if group == 1 else G2P
    pts = np.ascontiguousarray(points, dtype=dt)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    n = len(pts)
    limbs = sc.size // max(n, 1) if n else 1
    out = np.zeros(1, dtype=dt)
    outp = np.zeros(1, dtype=pdt)
    threads = threads or os.cpu_count() or 1
    getattr(r, f"ref_{g}_msm_pippenger")(_ptr(out), _ptr(outp), _ptr(pts), _ptr(sc), ctypes.c_int(limbs),
                                         ctypes.c_int64(n), ctypes.c_int(threads))
    return out, outp


def proj_to_affine(proj, group=1):
    dt, g = _grp(group)
    pdt = G1P if group == 1 else G2P
    p = np.ascontiguousarray(proj, dtype=pdt).reshape(-1)
    out = np.zeros(len(p), dtype=dt)
    fn = getattr(lib(), f"orc_{g}_proj_to_affine")
    for i in range(len(p)):
        fn(ctypes.c_void_p(out.ctypes.data + i * dt.itemsize), ctypes.c_void_p(p.ctypes.data + i * pdt.itemsize))
    return out


def on_curve(point, group=1) -> bool:
    dt, g = _grp(group)
    p = np.ascontiguousarray(point, dtype=dt).reshape(1)
    fn = getattr(lib(), f"orc_{g}_on_curve")
    fn.restype = ctypes.c_bool
    return bool(fn(_ptr(p)))


def same_point(a, b) -> bool:
    """Field-wise equality of affine points (pad bytes ignored)."""
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if bool(x["infinity"]) != bool(y["infinity"]):
            return False
        if not x["infinity"]:
            if not (np.array_equal(x["x"], y["x"]) and np.array_equal(x["y"], y["y"])):
                return False
    return True


def generator_multiple(s: int, group=1) -> np.ndarray:
    """(s mod r) * G in Montgomery-form canonical affine."""
    g = g1_generator() if group == 1 else g2_generator()
    return scalar_mul(g, s % R_ORDER, group=group)
