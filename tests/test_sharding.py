"""CPU: the sharded-MSM host logic over two gloo ranks.

Each rank computes the partial MSM of its slice (on the CPU with the oracle,
standing in for the device pipeline), the partials are exchanged with one
all_gather, and every rank adds them with the library's host-side projective
sum.  The result must equal the single-process MSM bit for bit (canonical
affine).  Also covers the slicing arithmetic.
"""
import os
import socket

import numpy as np
import pytest

from gpu_msm_b200.sharding import shard_range


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 64, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch
    import torch.distributed as dist

    import gpu_msm_b200 as gm
    import oracle
    from gpu_msm_b200 import sharding
    from gpu_msm_b200 import workload as wl
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sc = wl.make_scalars(n, seed=21)
        logs = wl.make_base_logs(n, seed=22)
        g = oracle.g1_generator()
        pts = np.concatenate([oracle.scalar_mul(g, t) for t in wl.limbs_to_ints(logs)])

        def local(b, e):
            aff = oracle.msm_pippenger(pts[b:e], sc[b:e], group=1, threads=2)
            proj = gm.affine_to_projective(aff, 1)
            return torch.from_numpy(proj.view(np.uint64).view(np.int64).reshape(-1).copy())

        res = sharding.sharded_msm(n, local, sharding.host_combine_g1, gm.G1P_WORDS)
        proj = res.numpy().view(np.uint64).view(gm.G1P)
        got = gm.projective_to_affine(proj, 1)
        want = oracle.msm_pippenger(pts, sc, group=1, threads=2)
        q.put((rank, bool(oracle.same_point(got, want))))
    finally:
        dist.destroy_process_group()


def test_sharded_msm_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 96, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    results = dict(q.get(timeout=10) for _ in range(2))
    assert results == {0: True, 1: True}
