"""CPU: the oracle's single-element semantics (oracle/pyref.py fp_elem,
fp2_elem, point_elem), pinned against the reference's own host functions
(oracle/_ref/libref.so, compiled from the reference sources) on the cases the
GPU parity test uses; and the Python op tables against the C header."""
import ctypes
import os
import re
import time

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from oracle import pyref
from tests import element_cases as ec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref():
    L = oracle.ref_lib()
    if L is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    for name in ("ref_fp_elem", "ref_fp2_elem"):
        getattr(L, name).argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 3 + [ctypes.c_uint64]
        getattr(L, name).restype = ctypes.c_int
    for name in ("ref_g1_point_elem", "ref_g2_point_elem"):
        getattr(L, name).argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_uint64]
        getattr(L, name).restype = ctypes.c_int
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def test_op_tables_match_header():
    """gm.FP_OPS / FP2_OPS / POINT_OPS list the ops in the order of the
    GM_FP_*, GM_FP2_* and GM_PT_* codes of include/gpu_msm_b200.h."""
    hdr = open(os.path.join(ROOT, "include", "gpu_msm_b200.h")).read()
    for prefix, ops in (("GM_FP_", gm.FP_OPS), ("GM_FP2_", gm.FP2_OPS), ("GM_PT_", gm.POINT_OPS)):
        codes = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(prefix + r"(\w+) = (\d+)", hdr)}
        assert codes.pop("op_count") == len(ops)
        names = {"to_mont": "to_mont", "from_mont": "from_mont", "is_qr": "is_qr"}
        for i, op in enumerate(ops):
            assert codes[names.get(op, op)] == i, (prefix, op)


def test_fp_elem_semantics_match_reference():
    L = _ref()
    for op, a, b, c, arg in ec.fp_cases():
        want, flag = pyref.fp_elem(op, a, b, c, arg)
        out, xa, xb = ec.fp_np(c), ec.fp_np(a), ec.fp_np(b)  # kept alive across the call
        got_flag = L.ref_fp_elem(op.encode(), _p(out), _p(xa), _p(xb), arg)
        assert got_flag != -99, op
        if want is not None:
            assert ec.fp_int(out) == want, (op, a, b, arg)
        if op in ("cmp", "is_zero", "is_one", "is_qr", "sqrt"):
            assert got_flag == flag, (op, a, b)


def test_fp2_elem_semantics_match_reference():
    L = _ref()
    for op, a, b, c, arg in ec.fp2_cases():
        want, flag = pyref.fp2_elem(op, a, b, c, arg)
        out, xa, xb = ec.fp2_np(c), ec.fp2_np(a), ec.fp2_np(b)
        got_flag = L.ref_fp2_elem(op.encode(), _p(out), _p(xa), _p(xb), arg)
        assert got_flag != -99, op
        if want is not None:
            assert ec.fp2_int(out) == want, (op, a, b)
        if op in ("cmp", "is_zero", "is_one"):
            assert got_flag == flag, (op, a, b)


@pytest.mark.parametrize("group", [1, 2])
def test_point_elem_semantics_match_reference(group):
    """Affine add / double / neg / conversions and double-and-add scalar
    multiplication (the reference's naive affine form: one inversion per
    step, so the full-width cases run on G1 only)."""
    L = _ref()
    fn = L.ref_g1_point_elem if group == 1 else L.ref_g2_point_elem
    t0 = time.time()
    for op, p, q, k, limbs in ec.point_cases(group, heavy=True):
        out, xp, xq = ec.point_np(None, group), ec.point_np(p, group), ec.point_np(q, group)
        ks = oracle.int_to_limbs(k, max(limbs, 1))
        rc = fn(op.encode(), _p(out), _p(xp), _p(xq), _p(ks), limbs, k & 0xFFFFFFFFFFFFFFFF)
        assert rc == 0, op
        assert ec.point_from_np(out, group) == ec.expected_point(op, p, q, k, limbs, group), (op, k)
    assert time.time() - t0 < 120
