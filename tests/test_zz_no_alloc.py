"""GPU: the allocation-free G1 MSM entry point (gm_g1_msm_device_noalloc).

Some callers cannot allocate device memory per call: a framework that gave
nearly all of HBM to its own caching allocator, or latency-critical code that
must not take the implicit synchronisation of cudaMalloc/cudaFree.  This entry
point serves them from a fixed workspace compiled into the library.  Its
results must equal the regular device entry point's (bit for bit, in
canonical affine coordinates) on consecutive calls that reuse the shared
workspace.  The file name makes pytest collect it last.
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


def test_noalloc_matches_regular_entry_point_on_consecutive_calls(cuda):
    import torch
    for call, (n, limbs, seed) in enumerate([(4096, 5, 11), (777, 1, 12), (4096, 5, 13)]):
        sc = wl.make_scalars(n, seed=seed)[:, :limbs].copy()
        logs = wl.make_base_logs(n, seed=seed + 100)
        pts = gm.generator_mul_batch(_dev(logs, cuda), group=1)
        sc_d = _dev(sc, cuda).reshape(n, limbs)
        out = torch.empty(gm.G1P_WORDS, dtype=torch.int64, device=cuda)
        rc = gm.lib().gm_g1_msm_device_noalloc(None, 0, ctypes.c_void_p(out.data_ptr()),
                                               ctypes.c_void_p(pts.data_ptr()), ctypes.c_void_p(sc_d.data_ptr()),
                                               limbs, n)
        assert rc == 0, gm.lib().gm_last_error()
        ref = gm.msm_device(pts, sc_d, group=1, stream=torch.cuda.default_stream())
        torch.cuda.synchronize()
        got_aff, ref_aff = _affine(out), _affine(ref)
        assert not got_aff[0]["infinity"]
        assert oracle.same_point(got_aff, ref_aff), f"call {call}"


def test_noalloc_rejects_requests_beyond_its_limit(cuda):
    import torch
    n = gm.NOALLOC_MAX_POINTS + 1
    pts = torch.zeros((n, gm.G1_WORDS), dtype=torch.int64, device=cuda)
    sc = torch.zeros((n, 5), dtype=torch.int64, device=cuda)
    out = torch.zeros(gm.G1P_WORDS, dtype=torch.int64, device=cuda)
    rc = gm.lib().gm_g1_msm_device_noalloc(None, 0, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(pts.data_ptr()),
                                           ctypes.c_void_p(sc.data_ptr()), 5, n)
    assert rc == -1
    assert b"4096" in gm.lib().gm_last_error()
