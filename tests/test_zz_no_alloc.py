"""GPU: the allocation-free G1 MSM entry point (gm_g1_msm_device_noalloc).

Some callers cannot allocate device memory per call: a framework that gave
nearly all of HBM to its own caching allocator, or latency-critical code that
must not take the implicit synchronisation of cudaMalloc/cudaFree.  This entry
point serves them from a fixed workspace compiled into the library.  On
consecutive calls that reuse that shared workspace, every result must be the
exact MSM (sum_i k_i t_i mod r) * G of its inputs (the bases are t_i * G) and
equal the regular device entry point's, bit for bit in canonical affine
coordinates, with the consistency flag clear.  The cases include the largest
request the limits accept (4096 points with 8 scalar limbs, 65 windows) and
skewed scalars whose buckets span many accumulation slices.  The file name
makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(cuda)


def _affine(out):
    return oracle.proj_to_affine(gm.to_numpy_proj(out, 1), 1)


def _scalars(n, limbs, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == "random":
        sc = wl.make_scalars(n, seed=seed)
        if limbs > 5:
            # full-width limbs: scalars far above r (the MSM reduces them mod r)
            sc = rng.integers(0, 2 ** 64, size=(n, limbs), dtype=np.uint64)
        return np.ascontiguousarray(sc[:, :limbs])
    sc = np.zeros((n, limbs), dtype=np.uint64)
    if kind == "all_equal":      # one bucket per window holds every point
        sc[:] = wl.make_scalars(1, seed=seed)[0, :limbs]
    elif kind == "all_one":      # every entry in bucket 0 of window 0
        sc[:, 0] = 1
    elif kind == "one_two":      # two buckets of n/2 entries each
        sc[: n // 2, 0] = 1
        sc[n // 2:, 0] = 2
    return sc


# consecutive calls, each reusing the workspace the previous one left behind
CASES = [
    (4096, 5, "random", 11),
    (777, 1, "random", 12),
    (4096, 8, "random", 13),     # largest accepted request: 65 windows of 8 bits
    (4096, 5, "all_equal", 14),
    (4096, 5, "all_one", 15),
    (4096, 8, "one_two", 16),
    (1, 5, "random", 17),
]


def test_noalloc_matches_oracle_and_regular_entry_point_on_consecutive_calls(cuda):
    import torch
    err = torch.full((1,), -1, dtype=torch.int32, device=cuda)
    for call, (n, limbs, kind, seed) in enumerate(CASES):
        sc = _scalars(n, limbs, kind, seed)
        logs = wl.make_base_logs(n, seed=seed + 100)
        pts = gm.generator_mul_batch(_dev(logs, cuda), group=1)
        sc_d = _dev(sc, cuda).reshape(n, limbs)
        out = torch.empty(gm.G1P_WORDS, dtype=torch.int64, device=cuda)
        err.fill_(-1)
        rc = gm.lib().gm_g1_msm_device_noalloc(None, 0, ctypes.c_void_p(out.data_ptr()),
                                               ctypes.c_void_p(pts.data_ptr()), ctypes.c_void_p(sc_d.data_ptr()),
                                               limbs, n, ctypes.c_void_p(err.data_ptr()))
        assert rc == 0, gm.lib().gm_last_error()
        ref = gm.msm_device(pts, sc_d, group=1, stream=torch.cuda.default_stream())
        torch.cuda.synchronize()
        assert int(err.item()) == 0, f"call {call}: consistency flag {int(err.item())}"
        got = _affine(out)
        want = oracle.generator_multiple(wl.expected_log(sc, logs))
        assert oracle.same_point(got, want), f"call {call} ({n}, {limbs}, {kind}) != (sum k t) G"
        assert oracle.same_point(got, _affine(ref)), f"call {call}: differs from gm_g1_msm_device"


def test_noalloc_small_case_against_reference_structured_pippenger(cuda):
    """A 64-point case against the oracle's reference-structured Pippenger,
    run straight after the largest request so the array holds stale data."""
    import torch
    n = 64
    sc = wl.make_scalars(n, seed=21)
    logs = wl.make_base_logs(n, seed=22)
    pts = gm.generator_mul_batch(_dev(logs, cuda), group=1)
    out = gm.msm_device_noalloc(pts, _dev(sc, cuda).reshape(n, 5))
    torch.cuda.synchronize()
    want = oracle.msm_pippenger(gm.to_numpy_points(pts, 1), sc, group=1)
    assert oracle.same_point(_affine(out), want)


def test_noalloc_rejects_requests_beyond_its_limit(cuda):
    import torch
    n = gm.NOALLOC_MAX_POINTS + 1
    pts = torch.zeros((n, gm.G1_WORDS), dtype=torch.int64, device=cuda)
    sc = torch.zeros((n, 5), dtype=torch.int64, device=cuda)
    out = torch.zeros(gm.G1P_WORDS, dtype=torch.int64, device=cuda)
    rc = gm.lib().gm_g1_msm_device_noalloc(None, 0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(pts.data_ptr()),
                                           ctypes.c_void_p(sc.data_ptr()), 5, n, None)
    assert rc == -1
    assert b"4096" in gm.lib().gm_last_error()
    sc9 = torch.zeros((16, 9), dtype=torch.int64, device=cuda)
    rc = gm.lib().gm_g1_msm_device_noalloc(None, 0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(pts.data_ptr()),
                                           ctypes.c_void_p(sc9.data_ptr()), 9, 16, None)
    assert rc == -1
