"""Batch-plan autotuner.

For each group and size class e = floor(log2 n), builds a batch of MSMs of
2^e points over a resident synthetic table and times the batched pipeline
(CUDA events, after a warm-up run) for
  1. each candidate window width c around the cost model (defaults for the rest);
  2. at the best c, the accumulation slices of the class in resident waves of
     threads (1, 2, 4: finer work items for the queued accumulation, more
     partials for the fix-up);
  3. at those, the pass-A sort tile in points per thread (2, 4, 8: 512, 1024
     or 2048 points per tile: fewer, larger tiles mean fewer counters to scan,
     smaller ones more blocks)
and records the fastest in ``window_table.json`` next to this file:

    {"g1": {"8": {"c": 7, "slice_waves": 1, "sort_ppt": 4}, ...}, "g2": {...},
     "device": "...", "points_per_class": N}

``gpu_msm_b200.tuned_params(group, n)`` reads it; batch plans use it for every
MSM whose parameters are not given.  Run on the target GPU:

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

        def run(c, waves, ppt):
            plan = gm.BatchPlan(table, sizes, offs, window_bits=np.full(count, c, dtype=np.int32),
                                tuning=np.tile(np.array([waves, ppt], dtype=np.int32), (count, 1)))
            t = _time_plan(plan, sc, reps)
            plan.close()
            return t

        model = gm.default_window(group, n, 5)
        cands = sorted(set(c for c in range(max(2, model - 3), min(20, model + 2) + 1)))
        t_c = {c: run(c, 1, 4) for c in cands}
        c = min(t_c, key=t_c.get)
        t_w = {w: (t_c[c] if w == 1 else run(c, w, 4)) for w in (1, 2, 4)}
        waves = min(t_w, key=t_w.get)
        t_p = {q: (t_w[waves] if q == 4 else run(c, waves, q)) for q in (2, 4, 8)}
        ppt = min(t_p, key=t_p.get)
        result[str(e)] = {"c": int(c), "slice_waves": int(waves), "sort_ppt": int(ppt)}
        detail[str(e)] = {"count": count, "model": model,
                          "ms_by_c": {str(k): round(v, 3) for k, v in t_c.items()},
                          "ms_by_slice_waves": {str(k): round(v, 3) for k, v in t_w.items()},
                          "ms_by_sort_ppt": {str(k): round(v, 3) for k, v in t_p.items()}}
        print(f"g{group} 2^{e:2d} x{count:4d}: c={c:2d} waves={waves} ppt={ppt} ({t_p[ppt]:.3f} ms; "
              f"c alone {t_c[c]:.3f} ms), cost model {model}", flush=True)
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
