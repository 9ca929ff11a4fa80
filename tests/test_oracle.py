"""CPU: pin the oracle before trusting it.

* the C restatement (oracle/oracle.c) against the golden vectors, which
  restate the reference's own known-answer tests (tests/test_fp.cu,
  tests/test_fp2.cu, tests/test_msm.cu) and pure-Python big-integer results;
* against the reference's own host code (oracle/_ref) when it was built;
* the derived constants: r*G = O on both groups, generators on the curves the
  points actually satisfy;
* the CPU configuration (G1, n = 1024): reference-structured Pippenger equals
  naive double-and-add bit for bit.
"""
import json
import os
import random

import numpy as np
import pytest

import oracle
from oracle import pyref
from gpu_msm_b200 import workload as wl

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def fp_arr(vals):
    return oracle.ints_to_fp_array([int(v, 16) for v in vals])


def fp2_arr(vals):
    out = np.zeros((len(vals), 2, 7), dtype=np.uint64)
    for i, v in enumerate(vals):
        out[i, 0] = oracle.int_to_limbs(int(v[0], 16))
        out[i, 1] = oracle.int_to_limbs(int(v[1], 16))
    return out


def test_constants():
    assert oracle.P == pyref.P
    assert pyref.R_ORDER.bit_length() == 299
    assert pyref.mul(pyref.g1(), pyref.R_ORDER, 1) is None
    assert pyref.mul(pyref.g2(), pyref.R_ORDER, 2) is None
    assert pyref.on_curve(pyref.g1(), 1) and pyref.on_curve(pyref.g2(), 2)
    assert oracle.on_curve(oracle.g1_generator(), 1)
    assert oracle.on_curve(oracle.g2_generator(), 2)
    # (r-1) * G = -G
    m = oracle.from_mont(oracle.scalar_mul(oracle.g1_generator(), pyref.R_ORDER - 1))[0]
    assert oracle.limbs_to_int(m["x"]) == pyref.G1_X
    assert oracle.limbs_to_int(m["y"]) == pyref.P - pyref.G1_Y


def test_field_kats():
    kats = load("field_kat.json")["kats"]
    by_op = {}
    for k in kats:
        by_op.setdefault(k["op"], []).append(k)
    for op, ks in by_op.items():
        if op.startswith("fp2"):
            a, b, c = fp2_arr([k["a"] for k in ks]), fp2_arr([k["b"] for k in ks]), fp2_arr([k["c"] for k in ks])
            got = {"fp2_mul": oracle.fp2_mul, "fp2_mont_mul": oracle.fp2_mont_mul}[op](a, b)
        else:
            a, b, c = fp_arr([k["a"] for k in ks]), fp_arr([k["b"] for k in ks]), fp_arr([k["c"] for k in ks])
            if op == "fp_add":
                got = np.stack([_c_add(x, y) for x, y in zip(a, b)])
            elif op == "fp_sub":
                got = np.stack([_c_sub(x, y) for x, y in zip(a, b)])
            else:
                got = {"fp_mul": oracle.fp_mul, "fp_mont_mul": oracle.fp_mont_mul}[op](a, b)
        assert np.array_equal(got, c), op


def _c_add(x, y):
    import ctypes
    out = np.zeros(7, dtype=np.uint64)
    x = np.ascontiguousarray(x)
    y = np.ascontiguousarray(y)
    oracle.lib().orc_fp_add(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(x.ctypes.data),
                            ctypes.c_void_p(y.ctypes.data))
    return out


def _c_sub(x, y):
    import ctypes
    out = np.zeros(7, dtype=np.uint64)
    x = np.ascontiguousarray(x)
    y = np.ascontiguousarray(y)
    oracle.lib().orc_fp_sub(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(x.ctypes.data),
                            ctypes.c_void_p(y.ctypes.data))
    return out


def golden_inputs(case):
    g = case["group"]
    gen = oracle.g1_generator() if g == 1 else oracle.g2_generator()
    pts = np.concatenate([oracle.scalar_mul(gen, int(k, 16) if isinstance(k, str) else k, group=g)
                          for k in case["bases_k"]])
    L = case["limbs"]
    sc = np.array([[(int(v, 16) >> (64 * j)) & (2 ** 64 - 1) for j in range(L)] for v in case["scalars"]],
                  dtype=np.uint64)
    return pts, sc


def matches_expected(aff_mont, case):
    g = case["group"]
    std = oracle.from_mont(aff_mont, group=g)[0]
    exp = case["expected"]
    if exp["infinity"]:
        return bool(std["infinity"])
    if std["infinity"]:
        return False
    if g == 1:
        return (oracle.limbs_to_int(std["x"]) == int(exp["x"], 16)
                and oracle.limbs_to_int(std["y"]) == int(exp["y"], 16))
    got = [oracle.limbs_to_int(std["x"][0]), oracle.limbs_to_int(std["x"][1]),
           oracle.limbs_to_int(std["y"][0]), oracle.limbs_to_int(std["y"][1])]
    return got == [int(v, 16) for v in exp["x"] + exp["y"]]


@pytest.mark.parametrize("case", load("msm_golden.json")["cases"], ids=lambda c: c["name"])
def test_msm_golden_c_oracle(case):
    pts, sc = golden_inputs(case)
    g = case["group"]
    assert matches_expected(oracle.msm_pippenger(pts, sc, group=g), case)
    assert matches_expected(oracle.msm_naive(pts, sc, group=g), case)


@pytest.mark.parametrize("case", load("msm_golden.json")["cases"], ids=lambda c: c["name"])
def test_msm_golden_reference_host(case):
    if oracle.ref_lib() is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    pts, sc = golden_inputs(case)
    aff, _ = oracle.ref_msm_pippenger(pts, sc, group=case["group"])
    assert matches_expected(aff, case)


def test_field_against_reference_host():
    ref = oracle.ref_lib()
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    import ctypes
    rng = random.Random(3)
    vals = [rng.randrange(pyref.P) for _ in range(256)] + [0, 1, pyref.P - 1]
    a = oracle.ints_to_fp_array(vals)
    b = oracle.ints_to_fp_array(vals[::-1])
    for name, fn in (("mont_mul", oracle.fp_mont_mul), ("mul", oracle.fp_mul)):
        want = np.zeros_like(a)
        getattr(ref, f"ref_fp_{name}_batch")(ctypes.c_void_p(want.ctypes.data), ctypes.c_void_p(a.ctypes.data),
                                             ctypes.c_void_p(b.ctypes.data), ctypes.c_int64(len(a)))
        assert np.array_equal(fn(a, b), want), name


def test_projective_ops_match_reference_host():
    """The oracle restates the reference's projective formulas exactly, so
    even the (non-unique) projective coordinates agree."""
    ref = oracle.ref_lib()
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    import ctypes
    g = oracle.g1_generator()
    rng = random.Random(11)
    pts = [oracle.scalar_mul(g, rng.randrange(1, pyref.R_ORDER)) for _ in range(8)]
    for i in range(len(pts) - 1):
        a = np.zeros(1, dtype=oracle.G1P)
        b = np.zeros(1, dtype=oracle.G1P)
        oracle.lib().orc_g1_affine_to_proj(ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(pts[i].ctypes.data))
        oracle.lib().orc_g1_affine_to_proj(ctypes.c_void_p(b.ctypes.data), ctypes.c_void_p(pts[i + 1].ctypes.data))
        mine = np.zeros(1, dtype=oracle.G1P)
        theirs = np.zeros(1, dtype=oracle.G1P)
        oracle.lib().orc_g1p_add(ctypes.c_void_p(mine.ctypes.data), ctypes.c_void_p(a.ctypes.data),
                                 ctypes.c_void_p(b.ctypes.data))
        ref.ref_g1p_add(ctypes.c_void_p(theirs.ctypes.data), ctypes.c_void_p(a.ctypes.data),
                        ctypes.c_void_p(b.ctypes.data))
        assert mine.tobytes() == theirs.tobytes()
        oracle.lib().orc_g1p_double(ctypes.c_void_p(mine.ctypes.data), ctypes.c_void_p(a.ctypes.data))
        ref.ref_g1p_double(ctypes.c_void_p(theirs.ctypes.data), ctypes.c_void_p(a.ctypes.data))
        assert mine.tobytes() == theirs.tobytes()


def test_cpu_config_pippenger_equals_naive():
    """Config 0: plain G1 MSM, n = 1024, scalars uniform in [0, r) with 1%
    zeros and 1% ones, bases k*G with 2% duplicates; Pippenger (reference
    structure) must equal naive double-and-add bit for bit."""
    from gpu_msm_b200 import workload
    n = 1024
    sc = workload.make_scalars(n, seed=42)
    logs = workload.make_base_logs(n, seed=4242)
    g = oracle.g1_generator()
    pts = np.concatenate([oracle.scalar_mul(g, t) for t in workload.limbs_to_ints(logs)])
    a = oracle.msm_pippenger(pts, sc)
    b = oracle.msm_naive(pts, sc)
    assert oracle.same_point(a, b)
    c = oracle.generator_multiple(workload.expected_log(sc, logs))
    assert oracle.same_point(a, c)


def test_fast_expected_log_matches_big_integers():
    """workload.dot_log (exact float64 limb-product sums) equals the plain
    big-integer sum_i k_i t_i mod r, for 1, 5 and 8 limbs and across the
    2^20-row chunk boundary."""
    rng = np.random.default_rng(3)
    for n, limbs in [(1, 5), (33, 1), (2000, 8), ((1 << 20) + 3, 5)]:
        sc = rng.integers(0, 2 ** 64, size=(n, limbs), dtype=np.uint64)
        logs = wl.make_base_logs(n, seed=n)
        assert wl.dot_log(wl.limbs16(sc), wl.limbs16(logs)) == wl.expected_log(sc, logs)
    sizes = np.array([5, 1, 300], dtype=np.int64)
    sc = wl.make_scalars(306, seed=4)
    logs = wl.make_base_logs(400, seed=5)
    offs = np.array([0, 7, 100])
    got = wl.expected_logs(sizes, sc, logs, offs)
    assert got == [wl.expected_log(sc[0:5], logs[0:5]), wl.expected_log(sc[5:6], logs[7:8]),
                   wl.expected_log(sc[6:306], logs[100:400])]
