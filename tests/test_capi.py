"""CPU: the C-ABI library loads, exports every symbol include/gpu_msm_b200.h
declares, runs its host-side helpers (which the reference also runs on the
CPU: rust-api/src/c_wrapper.cu:12-59, 261-288) bit-exactly against the oracle,
and fails loudly -- never falls back to a CPU path -- when no GPU is visible.
"""
import ctypes
import os
import random
import re

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from oracle import pyref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "gpu_msm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", txt, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "struct")))


def test_library_exports_every_declared_symbol():
    L = gm.lib()
    declared = header_functions()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert set(gm.C_API) <= set(declared)


def test_library_exports_reference_cxx_api():
    """Every mangled symbol of the reference's C++ MSM-path API (fixture made
    from the reference's own headers by golden/make_cxx_symbols.py) resolves
    in the library, so objects built against the reference's headers link."""
    L = gm.lib()
    path = os.path.join(ROOT, "tests", "golden", "cxx_symbols.txt")
    syms = [s.strip() for s in open(path) if s.strip() and not s.startswith("#")]
    assert len(syms) >= 120
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_host_arithmetic_selftest():
    """The host window combination's squaring and Jacobian doublings agree
    with the general product and the XYZZ formulas."""
    assert gm.lib().gm_host_selftest() == 0


def test_struct_sizes():
    assert (gm.G1.itemsize, gm.G2.itemsize, gm.G1P.itemsize, gm.G2P.itemsize) == (120, 232, 168, 336)


def rand_g1(rng, n):
    g = oracle.g1_generator()
    return np.concatenate([oracle.scalar_mul(g, rng.randrange(1, pyref.R_ORDER)) for _ in range(n)])


def rand_g2(rng, n):
    g = oracle.g2_generator()
    return np.concatenate([oracle.scalar_mul(g, rng.randrange(1, pyref.R_ORDER), group=2) for _ in range(n)])


def test_host_point_helpers_match_oracle():
    rng = random.Random(5)
    for group, pts in ((1, rand_g1(rng, 6)), (2, rand_g2(rng, 4))):
        proj = gm.affine_to_projective(pts, group)
        back = gm.projective_to_affine(proj, group)
        assert oracle.same_point(back, pts)
        # a non-trivial Z: the oracle's doubling output
        dbl = np.zeros(1, dtype=oracle.G1P if group == 1 else oracle.G2P)
        name = "orc_g1p_double" if group == 1 else "orc_g2p_double"
        getattr(oracle.lib(), name)(ctypes.c_void_p(dbl.ctypes.data), ctypes.c_void_p(proj[:1].ctypes.data))
        assert oracle.same_point(gm.projective_to_affine(dbl, group), oracle.proj_to_affine(dbl, group))
        assert oracle.same_point(gm.from_montgomery(pts, group), oracle.from_mont(pts, group))
    # infinity helpers
    inf = np.zeros(1, dtype=gm.G1)
    gm.lib().g1_point_at_infinity_wrapper(ctypes.c_void_p(inf.ctypes.data))
    assert gm.lib().g1_is_infinity_wrapper(ctypes.c_void_p(inf.ctypes.data))
    p = gm.affine_to_projective(inf, 1)
    assert not p["Z"].any()
    assert gm.projective_to_affine(p, 1)[0]["infinity"]


def test_fp_to_montgomery_wrapper():
    rng = random.Random(9)
    vals = [rng.randrange(pyref.P) for _ in range(32)] + [0, 1, pyref.P - 1]
    a = oracle.ints_to_fp_array(vals)
    assert np.array_equal(gm.fp_to_montgomery(a), oracle.fp_to_mont(a))


def test_msm_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    pts = rand_g1(random.Random(1), 2)
    with pytest.raises(gm.MSMError):
        gm.g1_msm(pts, np.array([[1], [2]], dtype=np.uint64))
    with pytest.raises(gm.MSMError):
        gm.g1_msm_wrapper(oracle.from_mont(pts), np.array([1, 2], dtype=np.uint64))


def test_reference_wrapper_rejects_nonpositive_n():
    out = np.zeros(1, dtype=gm.G1P)
    rc = gm.lib().g1_msm_wrapper(ctypes.c_void_p(out.ctypes.data), None, None, 0, 0)
    assert rc == -1  # c_wrapper.cu:71-73


def test_default_window_grows_with_n():
    ws = [gm.default_window(1, n, 5) for n in (16, 1 << 10, 1 << 16, 1 << 20)]
    assert ws == sorted(ws) and 3 <= ws[0] and ws[-1] <= 18
