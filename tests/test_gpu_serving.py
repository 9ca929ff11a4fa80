"""GPU: the continuous-batching server (gpu_msm_b200.serving), bit-exact.

Requests of both groups arrive while earlier batches run; every result must
be the same point as the request computed alone by a plain launch, and the
exact result (sum_j k_j t_j mod r) * G of its table slice.  Admission by
device memory must split batches under a small budget and reject a request
that cannot fit at all.
"""
import time

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import serving
from gpu_msm_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _tables(cuda, n1=1 << 12, n2=1 << 10):
    import torch
    out, logs = {}, {}
    for g, n, seed in ((1, n1, 81), (2, n2, 82)):
        lg = wl.make_base_logs(n, seed=seed)
        pts = gm.generator_mul_batch(torch.from_numpy(lg.view(np.int64)).to(cuda), group=g)
        out[g] = gm.ResidentBases(pts, group=g)
        logs[g] = lg
    return out, logs


def _canon(proj, group):
    return oracle.proj_to_affine(proj, group)


def test_serving_results_equal_alone_and_in_mix(cuda):
    import torch
    tables, logs = _tables(cuda)
    server = serving.MsmServer(tables, max_batch=16, max_points=1 << 14, slots=2).start()
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(40):
        g = 1 if rng.random() < 0.7 else 2
        n = int(2 ** rng.uniform(2, 10))
        sc = wl.make_scalars(n, seed=900 + i, one_frac=0.0)
        reqs.append((g, sc, server.submit(g, sc)))
        if i % 10 == 9:
            time.sleep(0.002)
    for _, _, r in reqs:
        assert r.done.wait(60)
    server.stop()
    assert max(b[2] for b in server.batches) > 1, "no batch held more than one request"
    for g, sc, r in reqs:
        assert r.error is None
        alone = tables[g].msm(torch.from_numpy(sc.view(np.int64)).to(cuda))
        torch.cuda.synchronize()
        got = _canon(r.result, g)
        assert oracle.same_point(got, _canon(gm.to_numpy_proj(alone, g), g))
        want = oracle.generator_multiple(wl.expected_log(sc, logs[g][:len(sc)]), group=g)
        assert oracle.same_point(got, want)


def test_serving_admission_by_memory(cuda):
    tables, logs = _tables(cuda, n1=1 << 14, n2=1 << 9)
    # slot workspaces that hold two 256-point requests but not three, and a
    # request that does not fit alone (workspace sizes follow the tuned window
    # widths, so both are derived from gm_batch_workspace_bytes)
    slot = gm.batch_workspace_bytes(tables[1], [256, 256])
    assert gm.batch_workspace_bytes(tables[1], [256] * 3) > slot
    big_n = next((n for n in (1024, 2048, 4096, 8192, 16384)
                  if gm.batch_workspace_bytes(tables[1], [n]) > slot), None)
    assert big_n is not None
    server = serving.MsmServer(tables, max_batch=32, max_points=1 << 14, slots=2, slot_bytes=slot).start()
    assert server.slot_bytes <= slot
    reqs = []
    for i in range(12):
        sc = wl.make_scalars(256, seed=700 + i, one_frac=0.0)
        reqs.append((sc, server.submit(1, sc)))
    big = server.submit(1, wl.make_scalars(big_n, seed=799))
    for _, r in reqs:
        assert r.done.wait(60)
    assert big.done.wait(60)
    server.stop()
    g1_batches = [b for b in server.batches if b[1] == 1]
    assert max(b[2] for b in g1_batches) <= 2, "a batch exceeded its slot's workspace"
    assert big.error is not None and "budget" in big.error
    for sc, r in reqs:
        want = oracle.generator_multiple(wl.expected_log(sc, logs[1][:len(sc)]), group=1)
        assert oracle.same_point(_canon(r.result, 1), want)
