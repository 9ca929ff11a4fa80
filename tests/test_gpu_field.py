"""GPU: Fp / Fp2 multiplication kernels against the oracle, bit-exact.

Covers the reference's field known-answer tests (golden/field_kat.json),
edge values (0, 1, p-1, p-2, R mod p, 2^445) and seeded random inputs, for
the Montgomery-form products (fp_mont_mul, fp2_mont_mul) and the normal-form
products behind fp_mul_array_device / fp2_mul_array_host.
"""
import json
import os
import random

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from oracle import pyref

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(cuda)


def host(t):
    return t.cpu().numpy().view(np.uint64)


def run(op, a, b, cuda):
    import torch
    ta, tb = dev(a, cuda), dev(b, cuda)
    out = gm.field_mul_array(ta.reshape(len(a), -1), tb.reshape(len(b), -1), op=op)
    torch.cuda.synchronize()
    return host(out).reshape(a.shape)


def test_golden_field_kats(cuda):
    kats = json.load(open(os.path.join(GOLD, "field_kat.json")))["kats"]
    for op in ("fp_mont_mul", "fp_mul"):
        ks = [k for k in kats if k["op"] == op]
        a = oracle.ints_to_fp_array([int(k["a"], 16) for k in ks])
        b = oracle.ints_to_fp_array([int(k["b"], 16) for k in ks])
        c = oracle.ints_to_fp_array([int(k["c"], 16) for k in ks])
        assert np.array_equal(run(op, a, b, cuda), c), op
    for op in ("fp2_mont_mul", "fp2_mul"):
        ks = [k for k in kats if k["op"] == op]

        def arr(key):
            out = np.zeros((len(ks), 2, 7), dtype=np.uint64)
            for i, k in enumerate(ks):
                out[i, 0] = oracle.int_to_limbs(int(k[key][0], 16))
                out[i, 1] = oracle.int_to_limbs(int(k[key][1], 16))
            return out
        assert np.array_equal(run(op, arr("a"), arr("b"), cuda), arr("c")), op


@pytest.mark.parametrize("n", [1, 255, 1 << 16])
def test_fp_mont_mul_random(cuda, n):
    rng = np.random.default_rng(n)
    vals = rng.integers(0, 2 ** 64, size=(n, 7), dtype=np.uint64)
    vals[:, 6] &= np.uint64(0x1FFFFFFFFFFFFFFF)  # < 2^445 < p
    a = vals
    b = np.roll(vals, 1, axis=0)
    assert np.array_equal(run("fp_mont_mul", a, b, cuda), oracle.fp_mont_mul(a, b))
    assert np.array_equal(run("fp_mul", a, b, cuda), oracle.fp_mul(a, b))


def test_fp_edges(cuda):
    P = pyref.P
    edge = [0, 1, 2, P - 1, P - 2, (1 << 448) % P, 1 << 445, P >> 1, (1 << 447) % P]
    rng = random.Random(1)
    edge += [rng.randrange(P) for _ in range(7)]
    xs = [x for x in edge for _ in edge]
    ys = [y for _ in edge for y in edge]
    a, b = oracle.ints_to_fp_array(xs), oracle.ints_to_fp_array(ys)
    assert np.array_equal(run("fp_mont_mul", a, b, cuda), oracle.fp_mont_mul(a, b))


def test_fp_mont_mul_limb52_patterns(cuda):
    """Structured operands: runs of ones, single high bits and values just
    below p at 52-bit strides (boundaries that do not line up with the 32-bit
    limbs of the product), against the oracle and the exact integer product,
    both orders, bit-exact."""
    P = pyref.P
    M = (1 << 52) - 1
    pats = [0, 1, M, 1 << 51, (1 << 52) - 2, P - 1, P - 2, P >> 1, (P + 1) // 2]
    for k in range(9):
        pats += [(1 << (52 * k)) - 1, 1 << (52 * k), (M << (52 * k)) % P, P - (1 << (52 * k))]
        pats += [sum(M << (52 * i) for i in range(k + 1)) % P]
    pats += [(1 << 446) - 1 if (1 << 446) - 1 < P else P - 7, ((1 << 416) - 1), (P >> 416) << 416]
    pats = sorted({v % P for v in pats})
    xs = [x for x in pats for _ in pats]
    ys = [y for _ in pats for y in pats]
    a, b = oracle.ints_to_fp_array(xs), oracle.ints_to_fp_array(ys)
    want = oracle.ints_to_fp_array([x * y * pow(1 << 448, -1, P) % P for x, y in zip(xs, ys)])
    assert np.array_equal(run("fp_mont_mul", a, b, cuda), want)
    assert np.array_equal(run("fp_mont_mul", a, b, cuda), oracle.fp_mont_mul(a, b))


def test_fp2_random(cuda):
    rng = np.random.default_rng(2)
    a = rng.integers(0, 2 ** 64, size=(4096, 2, 7), dtype=np.uint64)
    a[:, :, 6] &= np.uint64(0x1FFFFFFFFFFFFFFF)
    b = np.roll(a, 3, axis=0)
    assert np.array_equal(run("fp2_mont_mul", a, b, cuda), oracle.fp2_mont_mul(a, b))
    assert np.array_equal(run("fp2_mul", a, b, cuda), oracle.fp2_mul(a, b))


def test_fp_mont_mul_matches_reference_host(cuda):
    ref = oracle.ref_lib()
    if ref is None:
        pytest.skip("reference host code not built (oracle/_ref)")
    import ctypes
    rng = np.random.default_rng(3)
    a = rng.integers(0, 2 ** 64, size=(2048, 7), dtype=np.uint64)
    a[:, 6] &= np.uint64(0x1FFFFFFFFFFFFFFF)
    b = np.roll(a, 5, axis=0)
    want = np.zeros_like(a)
    ref.ref_fp_mont_mul_batch(ctypes.c_void_p(want.ctypes.data), ctypes.c_void_p(a.ctypes.data),
                              ctypes.c_void_p(b.ctypes.data), ctypes.c_int64(len(a)))
    assert np.array_equal(run("fp_mont_mul", a, b, cuda), want)


def test_fp_mont_sqr_matches_mul(cuda):
    """The dedicated squaring equals fp_mont_mul(a, a) of the oracle on edge
    values and seeded random elements."""
    import torch
    P = pyref.P
    edge = [0, 1, 2, 3, P - 1, P - 2, P - 3, (1 << 448) % P, 1 << 445, (1 << 446) - 1 if (1 << 446) - 1 < P else P - 5,
            P >> 1, (P >> 1) + 1, (1 << 447) % P, (1 << 32) - 1, (1 << 224) - 1]
    rng = random.Random(7)
    edge += [rng.randrange(P) for _ in range(4096)]
    a = oracle.ints_to_fp_array(edge)
    out = gm.field_sqr_array(dev(a, cuda).reshape(len(edge), -1))
    torch.cuda.synchronize()
    assert np.array_equal(host(out).reshape(a.shape), oracle.fp_mont_mul(a, a))
