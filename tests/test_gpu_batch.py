"""GPU: batched MSMs over a resident base table (gm_batch_plan_*), bit-exact.

Every output of a batch must equal the exact result (sum_i k_i t_i mod r) * G
of its own slice of the table (bases are t_i * G), and the plain single-MSM
launch over the same slice; with mixed window-width classes, with the plan
reused for new scalars, with the run captured in a CUDA graph and replayed,
and for G2.
"""
import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import workload as wl

pytestmark = pytest.mark.gpu


def t_dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(cuda)


def make_table(n, group, cuda, seed):
    logs = wl.make_base_logs(n, seed=seed)
    pts = gm.generator_mul_batch(t_dev(logs, cuda), group=group)
    return gm.ResidentBases(pts, group=group), logs


def batch_inputs(n_table, count, lo, hi, seed):
    sizes = np.minimum(wl.mixed_sizes(count, lo, hi, seed=seed), n_table)
    rng = np.random.default_rng(seed + 1)
    offs = np.array([rng.integers(0, n_table - s + 1) for s in sizes], dtype=np.int64)
    sc = wl.make_scalars(int(sizes.sum()), seed=seed + 2)
    return sizes, offs, sc


def expected(sizes, offs, sc, logs, group):
    out, row = [], 0
    for s, o in zip(sizes, offs):
        out.append(oracle.generator_multiple(wl.expected_log(sc[row:row + s], logs[o:o + s]), group=group))
        row += s
    return out


def check(res_t, want, group):
    got = gm.to_numpy_proj(res_t, group)
    for i, w in enumerate(want):
        assert oracle.same_point(oracle.proj_to_affine(got[i:i + 1], group), w), f"msm {i}"


def test_batch_g1_matches_oracle_and_plain(cuda):
    import torch
    table, logs = make_table(1 << 12, 1, cuda, seed=31)
    sizes, offs, sc = batch_inputs(1 << 12, 40, 2, 12, seed=32)
    plan = gm.BatchPlan(table, sizes, offs)
    sc_d = t_dev(sc, cuda).reshape(-1, 5)
    res = plan.run(sc_d)
    torch.cuda.synchronize()
    want = expected(sizes, offs, sc, logs, 1)
    check(res, want, 1)
    # plain launches over the same slices
    row = 0
    for i, (s, o) in enumerate(zip(sizes, offs)):
        one = table.msm(sc_d[row:row + s], offset=int(o))
        torch.cuda.synchronize()
        assert oracle.same_point(oracle.proj_to_affine(gm.to_numpy_proj(one, 1), 1), want[i])
        row += s
    # reuse of the plan with new scalars
    sc2 = wl.make_scalars(int(sizes.sum()), seed=99)
    res2 = plan.run(t_dev(sc2, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    check(res2, expected(sizes, offs, sc2, logs, 1), 1)
    plan.close()
    table.close()


def test_batch_mixed_window_classes(cuda):
    import torch
    table, logs = make_table(1 << 11, 1, cuda, seed=41)
    sizes, offs, sc = batch_inputs(1 << 11, 24, 1, 11, seed=42)
    wins = np.array([[3, 7, 11][i % 3] for i in range(len(sizes))], dtype=np.int32)
    plan = gm.BatchPlan(table, sizes, offs, window_bits=wins)
    assert sorted(w for w, _ in plan.classes()) == [3, 7, 11]
    res = plan.run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    want = expected(sizes, offs, sc, logs, 1)
    check(res, want, 1)
    plan.set_queue(False)
    res_q = plan.run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    check(res_q, want, 1)
    assert torch.equal(res_q, res)


def test_batch_tuning_parameters_keep_results(cuda):
    """Every (slice waves, sort tile) pair the autotuner may pick gives the
    exact result of every MSM in both accumulation modes (the slicing changes
    the order of the bucket sums, so the affine form is compared), and values
    outside {1,2,4} x {2,4,8} are rejected at plan creation."""
    import torch
    table, logs = make_table(1 << 12, 1, cuda, seed=45)
    sizes, offs, sc = batch_inputs(1 << 12, 20, 3, 12, seed=46)
    wins = np.array([[5, 9][i % 2] for i in range(len(sizes))], dtype=np.int32)
    want = expected(sizes, offs, sc, logs, 1)
    sc_d = t_dev(sc, cuda).reshape(-1, 5)
    for waves in (1, 2, 4):
        for ppt in (2, 4, 8):
            tun = np.tile(np.array([waves, ppt], dtype=np.int32), (len(sizes), 1))
            plan = gm.BatchPlan(table, sizes, offs, window_bits=wins, tuning=tun)
            for queue in (True, False):
                plan.set_queue(queue)
                res = plan.run(sc_d)
                torch.cuda.synchronize()
                check(res, want, 1)
    for bad in ([3, 4], [1, 16], [-1, 4]):
        tun = np.tile(np.array(bad, dtype=np.int32), (len(sizes), 1))
        with pytest.raises(gm.MSMError):
            gm.BatchPlan(table, sizes, offs, window_bits=wins, tuning=tun)


def test_batch_graph_capture_replay(cuda):
    import torch
    table, logs = make_table(1 << 11, 1, cuda, seed=51)
    sizes, offs, sc = batch_inputs(1 << 11, 16, 4, 11, seed=52)
    plan = gm.BatchPlan(table, sizes, offs, window_bits=[[6, 9][i % 2] for i in range(len(sizes))])
    static_sc = t_dev(sc, cuda).reshape(-1, 5).clone()
    out = torch.empty((len(sizes), gm.G1P_WORDS), dtype=torch.int64, device=cuda)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.run(static_sc, out=out)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        plan.run(static_sc, out=out)
    for seed in (53, 54):
        new = wl.make_scalars(int(sizes.sum()), seed=seed)
        static_sc.copy_(t_dev(new, cuda).reshape(-1, 5))
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        check(out, expected(sizes, offs, new, logs, 1), 1)
    del g


def test_batch_run_in_caller_workspace(cuda):
    """gm_batch_run_ws: the transient batch in a caller-owned workspace of
    gm_batch_workspace_bytes gives the exact results, the same words as the
    pooled gm_batch_run, and the workspace is reusable right away on the
    same stream; a workspace one byte short, or not 256-byte aligned, is
    refused before anything is enqueued."""
    import torch
    table, logs = make_table(1 << 11, 1, cuda, seed=47)
    table.precompute(8)
    sizes, offs, sc = batch_inputs(1 << 11, 18, 2, 11, seed=48)
    wins = np.array([[0, 5, 9][i % 3] for i in range(len(sizes))], dtype=np.int32)
    need = gm.batch_workspace_bytes(table, sizes, window_bits=wins)
    ws = torch.empty(need, dtype=torch.uint8, device=cuda)
    sc_d = t_dev(sc, cuda).reshape(-1, 5)
    want = expected(sizes, offs, sc, logs, 1)
    pooled = gm.batch_run(table, sizes, sc_d, base_offsets=offs, window_bits=wins)
    own = gm.batch_run(table, sizes, sc_d, base_offsets=offs, window_bits=wins, workspace=ws)
    torch.cuda.synchronize()
    check(own, want, 1)
    assert torch.equal(own, pooled)
    sc2 = wl.make_scalars(int(sizes.sum()), seed=49)
    again = gm.batch_run(table, sizes, t_dev(sc2, cuda).reshape(-1, 5), base_offsets=offs, window_bits=wins,
                         workspace=ws)
    torch.cuda.synchronize()
    check(again, expected(sizes, offs, sc2, logs, 1), 1)
    with pytest.raises(gm.MSMError):
        gm.batch_run(table, sizes, sc_d, base_offsets=offs, window_bits=wins, workspace=ws[:need - 1])
    with pytest.raises(gm.MSMError):
        gm.batch_run(table, sizes, sc_d, base_offsets=offs, window_bits=wins, workspace=ws[16:])


def test_batch_g2(cuda):
    import torch
    table, logs = make_table(1 << 9, 2, cuda, seed=61)
    sizes, offs, sc = batch_inputs(1 << 9, 8, 2, 9, seed=62)
    plan = gm.BatchPlan(table, sizes, offs)
    res = plan.run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    check(res, expected(sizes, offs, sc, logs, 2), 2)


def test_batch_precomputed_tables(cuda):
    """Fixed-base window tables: batches whose width has a table run with one
    bucket set per MSM; mixed with a width that has no table; results equal
    the oracle and the plain launches."""
    import torch
    table, logs = make_table(1 << 11, 1, cuda, seed=71)
    table.precompute(8).precompute(11)
    sizes, offs, sc = batch_inputs(1 << 11, 30, 1, 11, seed=72)
    # widths chosen by the library among the tables
    plan = gm.BatchPlan(table, sizes, offs)
    assert set(w for w, _ in plan.classes()) <= {8, 11}
    res = plan.run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    want = expected(sizes, offs, sc, logs, 1)
    check(res, want, 1)
    # explicit widths: 8 and 11 use tables, 5 does not
    wins = np.array([[5, 8, 11][i % 3] for i in range(len(sizes))], dtype=np.int32)
    plan2 = gm.BatchPlan(table, sizes, offs, window_bits=wins)
    res2 = plan2.run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    check(res2, want, 1)
    # single resident MSM through the table
    sc_d = t_dev(sc, cuda).reshape(-1, 5)
    one = table.msm(sc_d[:int(sizes[0])], offset=int(offs[0]))
    torch.cuda.synchronize()
    assert oracle.same_point(oracle.proj_to_affine(gm.to_numpy_proj(one, 1), 1), want[0])
    # graph capture and replay with new scalars
    static_sc = sc_d.clone()
    out = torch.empty((len(sizes), gm.G1P_WORDS), dtype=torch.int64, device=cuda)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.run(static_sc, out=out)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        plan.run(static_sc, out=out)
    new = wl.make_scalars(int(sizes.sum()), seed=73)
    static_sc.copy_(t_dev(new, cuda).reshape(-1, 5))
    g.replay()
    torch.cuda.synchronize()
    check(out, expected(sizes, offs, new, logs, 1), 1)
    del g


def test_batch_precomputed_heavy_and_infinity(cuda):
    """Precomputed tables with infinity bases in the set and scalars that put
    thousands of entries into a few buckets."""
    import torch
    n = 1 << 10
    logs = wl.make_base_logs(n, seed=81)
    pts = gm.generator_mul_batch(t_dev(logs, cuda), group=1)
    host = gm.to_numpy_points(pts, 1).copy()
    host["infinity"][::7] = 1
    table = gm.ResidentBases(t_dev(host, cuda).reshape(n, -1), group=1)
    table.precompute(9)
    sizes = np.array([n, 500, 77], dtype=np.int64)
    offs = np.array([0, 100, 900], dtype=np.int64)
    sc = wl.make_scalars(int(sizes.sum()), seed=82)
    sc[: n // 2] = 0
    sc[: n // 2, 0] = 1
    res = gm.batch_run(table, sizes, t_dev(sc, cuda).reshape(-1, 5), base_offsets=offs)
    torch.cuda.synchronize()
    got = gm.to_numpy_proj(res, 1)
    row = 0
    for i, (s_, o) in enumerate(zip(sizes, offs)):
        want = oracle.msm_pippenger(host[o:o + s_], sc[row:row + s_], group=1)
        assert oracle.same_point(oracle.proj_to_affine(got[i:i + 1], 1), want), i
        row += s_


def test_batch_precomputed_g2(cuda):
    import torch
    table, logs = make_table(1 << 9, 2, cuda, seed=91)
    table.precompute(7)
    sizes, offs, sc = batch_inputs(1 << 9, 8, 2, 9, seed=92)
    res = gm.BatchPlan(table, sizes, offs).run(t_dev(sc, cuda).reshape(-1, 5))
    torch.cuda.synchronize()
    check(res, expected(sizes, offs, sc, logs, 2), 2)


def _generator_multiples(logs_list, group):
    """(s mod r) * G for every s, from the oracle, in parallel (the oracle's C
    calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=8) as ex:
        return list(ex.map(lambda s: oracle.generator_multiple(s, group=group), logs_list))


def _check_all(res_t, sizes, sc, logs, group=1):
    want = _generator_multiples(wl.expected_logs(sizes, sc, logs), group)
    got = gm.to_numpy_proj(res_t, group)
    bad = [i for i, w in enumerate(want) if not oracle.same_point(oracle.proj_to_affine(got[i:i + 1], group), w)]
    assert not bad, f"{len(bad)} of {len(want)} outputs differ, first {bad[:5]}"


def test_batch_512_config_every_output(cuda):
    """The batched benchmark configuration exactly: 512 G1 MSMs of sizes
    floor(2^U), U ~ U[8, 16] (seed 7), each with its own scalars over a prefix
    of one resident 2^16-point table; window widths from the autotuner's
    table; the plan captured in a CUDA graph and replayed.  Every one of the
    512 outputs equals (sum_i k_i t_i mod r) * G, on two replays with
    different scalars, without and with fixed-base window tables."""
    import torch
    n_table, count = 1 << 16, 512
    table, logs = make_table(n_table, 1, cuda, seed=7070)
    sizes = wl.mixed_sizes(count, 8, 16, seed=7)
    total = int(sizes.sum())
    static_sc = torch.empty((total, 5), dtype=torch.int64, device=cuda)
    out = torch.empty((count, gm.G1P_WORDS), dtype=torch.int64, device=cuda)

    def graph_of(plan):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            plan.run(static_sc, out=out)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            plan.run(static_sc, out=out)
        return g

    sc0 = wl.make_scalars(total, seed=7171)
    static_sc.copy_(t_dev(sc0, cuda).reshape(-1, 5))
    plan = gm.BatchPlan(table, sizes)
    assert len(plan.classes()) > 1
    g = graph_of(plan)
    for seed in (7171, 7272):
        sc = wl.make_scalars(total, seed=seed)
        static_sc.copy_(t_dev(sc, cuda).reshape(-1, 5))
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        _check_all(out, sizes, sc, logs)
    del g
    # the same plan with one pipeline per class (the other accumulation mode)
    plan.set_queue(False)
    first = None
    g = graph_of(plan)
    for seed in (7575, 7575):
        sc = wl.make_scalars(total, seed=seed)
        static_sc.copy_(t_dev(sc, cuda).reshape(-1, 5))
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        _check_all(out, sizes, sc, logs)
        # deterministic whatever order the queue hands out the work
        if first is None:
            first = out.clone()
        else:
            assert torch.equal(out, first)
    del g
    plan.close()
    for c in (8, 10, 12, 14, 16):
        table.precompute(c)
    plan = gm.BatchPlan(table, sizes)
    for queue in (True, False):
        plan.set_queue(queue)
        g = graph_of(plan)
        for seed in (7373, 7474):
            sc = wl.make_scalars(total, seed=seed)
            static_sc.copy_(t_dev(sc, cuda).reshape(-1, 5))
            out.zero_()
            g.replay()
            torch.cuda.synchronize()
            _check_all(out, sizes, sc, logs)
        del g
    plan.close()
    table.close()
