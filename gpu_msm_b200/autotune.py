"""Window-width autotuner.

For each group and size class e = floor(log2 n), builds a batch of MSMs of
2^e points over a resident synthetic table, times the batched pipeline for
each candidate window width c (CUDA events, after a warm-up run) and records
the fastest in ``window_table.json`` next to this file:

    {"g1": {"8": 7, ...}, "g2": {...}, "device": "...", "points_per_class": N}

``gpu_msm_b200.tuned_window(group, n)`` reads it; batch plans use it for
every MSM whose window width is not given.  Run on the target GPU:

    python -m gpu_msm_b200.autotune [--quick]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "window_table.json")


def _time_plan(plan, sc, reps):
    import torch
    plan.run(sc)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        plan.run(sc)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune_group(group, lo, hi, points_per_class, reps, dev):
    import torch

    import gpu_msm_b200 as gm
    from gpu_msm_b200 import workload as wl
    n_table = 1 << hi
    logs = wl.make_base_logs(n_table, seed=777 + group)
    pts = gm.generator_mul_batch(torch.from_numpy(logs.view(np.int64)).to(dev), group=group)
    table = gm.ResidentBases(pts, group=group)
    del pts
    result, detail = {}, {}
    for e in range(lo, hi + 1):
        n = 1 << e
        count = max(1, min(512, points_per_class // n))
        sizes = np.full(count, n, dtype=np.int64)
        rng = np.random.default_rng(e)
        offs = rng.integers(0, n_table - n + 1, size=count).astype(np.int64)
        sc = torch.from_numpy(wl.make_scalars(count * n, seed=1000 + e).view(np.int64)).to(dev)
        model = gm.default_window(group, n, 5)
        cands = sorted(set(c for c in range(max(2, model - 3), min(20, model + 2) + 1)))
        times = {}
        for c in cands:
            plan = gm.BatchPlan(table, sizes, offs, window_bits=np.full(count, c, dtype=np.int32))
            times[c] = _time_plan(plan, sc, reps)
            plan.close()
        best = min(times, key=times.get)
        result[str(e)] = int(best)
        detail[str(e)] = {"count": count, "ms": {str(c): round(t, 3) for c, t in times.items()}, "model": model}
        print(f"g{group} 2^{e:2d} x{count:4d}: best c={best:2d} ({times[best]:.3f} ms), cost model {model}",
              flush=True)
    table.close()
    return result, detail


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="fewer classes and repetitions")
    ap.add_argument("--out", default=TABLE)
    args = ap.parse_args()
    dev = torch.device("cuda", 0)
    reps = 2 if args.quick else 3
    ppc = 1 << (17 if args.quick else 18)
    t0 = time.time()
    g1, d1 = tune_group(1, 4, 20, ppc, reps, dev)
    g2, d2 = tune_group(2, 4, 18, ppc, reps, dev)
    out = {"g1": g1, "g2": g2, "device": torch.cuda.get_device_name(0), "points_per_class": ppc,
           "detail": {"g1": d1, "g2": d2}, "seconds": round(time.time() - t0, 1)}
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
