"""MSM sharded over ranks (one process per GPU, torch.distributed).

An MSM  sum_i k_i P_i  splits by points: rank r of W takes the contiguous
slice ``shard_range(n, W, r)``, runs the whole single-GPU pipeline on it and
produces one projective partial sum.  The only exchange is one all_gather of
the W partials (168 B each for G1), after which every rank adds them
(``sum_projective`` on the device, or ``sum_projective_host``).  No kernel
reads another GPU's memory.

``sharded_msm`` takes the local MSM and the combine as arguments so the same
host logic runs with the CUDA library over NCCL and, in tests, with CPU
stand-ins over gloo.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, world: int, rank: int):
    """[begin, end) of rank's slice: contiguous, sizes differ by at most 1."""
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def sharded_msm(n: int, local_msm, combine, group_words: int, device=None, process_group=None):
    """local_msm(begin, end) -> int64 tensor (group_words,) partial sum of the
    rank's slice; combine(int64 tensor (world, group_words)) -> result.
    Returns the full MSM on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(process_group)
    rank = dist.get_rank(process_group)
    b, e = shard_range(n, world, rank)
    part = local_msm(b, e).reshape(group_words).to(torch.int64)
    if device is not None:
        part = part.to(device)
    gathered = torch.empty(world * group_words, dtype=torch.int64, device=part.device)
    dist.all_gather_into_tensor(gathered, part.contiguous(), group=process_group)
    return combine(gathered.view(world, group_words))


def device_local_msm(points, scalars, group: int = 1):
    """local_msm for the CUDA library: MSM of points[b:e] with scalars[b:e]
    (device tensors in the reference layout)."""
    import gpu_msm_b200 as gm

    def run(b, e):
        return gm.msm_device(points[b:e], scalars[b:e], group=group)
    return run


def device_combine(group: int = 1):
    import gpu_msm_b200 as gm

    def run(gathered):
        return gm.sum_projective(gathered, group=group)
    return run


def host_combine_g1(gathered):
    """combine on the CPU with the library's host arithmetic (G1)."""
    import torch

    import gpu_msm_b200 as gm
    arr = gathered.cpu().numpy().view(np.uint64).view(gm.G1P).reshape(-1)
    out = gm.sum_projective_host(arr)
    return torch.from_numpy(out.view(np.uint64).view(np.int64).reshape(-1).copy())
