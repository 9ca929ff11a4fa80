"""GPU: the device pieces of the sharded MSM on one B200.

* The partial MSMs of contiguous slices (``shard_range``), added with the
  device projective sum (``gm_g1_sum_projective``), give the full MSM: the
  exact result (sum_i k_i t_i mod r) * G of bases t_i * G, for 1 to 5 slices.
* ``sharded_msm`` over a one-rank NCCL process group, in a spawned child,
  runs the whole path of ``bench.py --gpus N`` (local MSM on the device, one
  all_gather, device combine) and gives the same point.  More ranks need
  more GPUs; their host logic is covered over gloo in test_sharding.py.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import sharding
from gpu_msm_b200 import workload as wl

pytestmark = pytest.mark.gpu

N = 5000


def _inputs(cuda):
    import torch
    sc = wl.make_scalars(N, seed=31)
    logs = wl.make_base_logs(N, seed=32)
    pts = gm.generator_mul_batch(torch.from_numpy(logs.view(np.int64)).to(cuda), group=1)
    want = oracle.generator_multiple(wl.expected_log(sc, logs), group=1)
    return pts, torch.from_numpy(sc.view(np.int64)).to(cuda), want


def _affine(proj_t):
    return oracle.proj_to_affine(gm.to_numpy_proj(proj_t.reshape(1, -1), 1), 1)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_slice_partials_add_up_on_the_device(cuda, world):
    import torch
    pts, sc, want = _inputs(cuda)
    local = sharding.device_local_msm(pts, sc, group=1)
    parts = torch.stack([local(*sharding.shard_range(N, world, r)).reshape(-1) for r in range(world)])
    total = sharding.device_combine(1)(parts)
    torch.cuda.synchronize()
    assert oracle.same_point(_affine(total), want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _nccl_worker(port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=dev)
    try:
        pts, sc, _ = _inputs(dev)
        res = sharding.sharded_msm(N, sharding.device_local_msm(pts, sc, group=1), sharding.device_combine(1),
                                   gm.G1P_WORDS, device=dev)
        torch.cuda.synchronize()
        q.put(gm.to_numpy_proj(res.reshape(1, -1), 1).tobytes())
    finally:
        dist.destroy_process_group()


def test_sharded_msm_over_one_nccl_rank(cuda):
    import multiprocessing as mp
    _, _, want = _inputs(cuda)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_worker, args=(_free_port(), q))
    p.start()
    p.join(240)
    if p.is_alive():
        p.kill()
        p.join()
    assert p.exitcode == 0
    proj = np.frombuffer(q.get(timeout=10), dtype=gm.G1P)
    assert oracle.same_point(oracle.proj_to_affine(proj, 1), want)
