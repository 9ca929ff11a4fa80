"""GPU: MSM parity, bit-exact in canonical affine coordinates.

Against the oracle on the same seeded inputs:
* golden fixtures (reference relation tests sum i*G, random cases with zeros,
  ones, duplicated bases and a cancelling P/-P pair);
* the reference's u64 C-ABI conventions (g1 points standard form, g2 points
  Montgomery form) through g1_msm_wrapper / g2_msm_wrapper;
* random MSMs over a sweep of sizes and window widths, infinity bases,
  all-equal bases, full-width scalars;
* the benchmark workloads: a 2^12 prefix of the G1 2^20 workload against the
  reference-structured CPU Pippenger (the reference's own host code when
  built), 64 sub-MSMs of 16 points against naive double-and-add, a 2^10 G2
  prefix, and the full G1 2^20 / G2 2^18 MSMs through the exact relation
  MSM = (sum_i k_i t_i mod r) * G (bases are t_i * G).
"""
import json
import os

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import workload as wl
from oracle import pyref

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def t_dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(cuda)


def make_bases(logs, group, cuda):
    """Bases t_i * G on the device (Montgomery, reference layout)."""
    import torch
    pts = gm.generator_mul_batch(t_dev(logs, cuda), group=group)
    torch.cuda.synchronize()
    return pts


def device_msm(pts, sc, group, cuda, c=0):
    import torch
    sc_t = sc if isinstance(sc, torch.Tensor) else t_dev(sc, cuda)
    out = gm.msm_device(pts, sc_t, group=group, window_bits=c)
    torch.cuda.synchronize()
    return oracle.proj_to_affine(gm.to_numpy_proj(out, group), group)


def check_bases_sample(pts, logs, group, k=8):
    host = gm.to_numpy_points(pts, group)
    gen = oracle.g1_generator() if group == 1 else oracle.g2_generator()
    idx = np.linspace(0, len(host) - 1, k).astype(int)
    for i in idx:
        want = oracle.scalar_mul(gen, wl.limbs_to_ints(logs[i:i + 1])[0], group=group)
        assert oracle.same_point(host[i:i + 1], want), i


def golden_cases():
    return json.load(open(os.path.join(GOLD, "msm_golden.json")))["cases"]


def expected_point(case):
    g = case["group"]
    exp = case["expected"]
    dt = oracle.G1 if g == 1 else oracle.G2
    out = np.zeros(1, dtype=dt)
    if exp["infinity"]:
        out["infinity"] = True
        return out
    if g == 1:
        out["x"][0] = oracle.int_to_limbs(int(exp["x"], 16))
        out["y"][0] = oracle.int_to_limbs(int(exp["y"], 16))
    else:
        for j in range(2):
            out["x"][0][j] = oracle.int_to_limbs(int(exp["x"][j], 16))
            out["y"][0][j] = oracle.int_to_limbs(int(exp["y"][j], 16))
    return oracle.to_mont(out, g)


def golden_inputs(case):
    L = case["limbs"]
    logs = np.array([oracle.int_to_limbs(int(k, 16) if isinstance(k, str) else k, 5) for k in case["bases_k"]])
    sc = np.array([[(int(v, 16) >> (64 * j)) & (2 ** 64 - 1) for j in range(L)] for v in case["scalars"]],
                  dtype=np.uint64)
    return logs, sc


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_golden_device_and_host_api(cuda, case):
    g = case["group"]
    logs, sc = golden_inputs(case)
    pts = make_bases(logs, g, cuda)
    want = expected_point(case)
    assert oracle.same_point(device_msm(pts, sc, g, cuda), want)
    host_pts = gm.to_numpy_points(pts, g)
    got = gm.msm(host_pts, sc, group=g, montgomery=True)
    assert oracle.same_point(oracle.proj_to_affine(got, g), want)
    assert oracle.same_point(gm.projective_to_affine(got, g), want)


def test_reference_u64_wrappers(cuda):
    """tests/test_msm.cu relations through the reference C-ABI conventions."""
    for N in (10, 100):
        g = oracle.g1_generator(mont=False)
        pts = np.repeat(g, N)
        sc = np.arange(1, N + 1, dtype=np.uint64)
        res = gm.g1_msm_wrapper(pts, sc)  # standard-form input (c_wrapper.cu:127)
        want = oracle.scalar_mul(oracle.g1_generator(), N * (N + 1) // 2)
        assert oracle.same_point(gm.projective_to_affine(res, 1), want)
    g2 = oracle.g2_generator()  # Montgomery-form input (c_wrapper.cu:223)
    res = gm.g2_msm_wrapper(np.repeat(g2, 10), np.arange(1, 11, dtype=np.uint64))
    want = oracle.scalar_mul(g2, 55, group=2)
    assert oracle.same_point(gm.projective_to_affine(res, 2), want)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 300, 1000])
def test_random_sizes_g1(cuda, n):
    sc = wl.make_scalars(n, seed=n)
    logs = wl.make_base_logs(n, seed=n + 1)
    pts = make_bases(logs, 1, cuda)
    got = device_msm(pts, sc, 1, cuda)
    host = gm.to_numpy_points(pts, 1)
    assert oracle.same_point(got, oracle.msm_pippenger(host, sc, group=1))
    assert oracle.same_point(got, oracle.generator_multiple(wl.expected_log(sc, logs)))


@pytest.mark.parametrize("c", [2, 3, 5, 8, 9, 10, 11, 13, 16, 17, 18, 20])
def test_window_sweep(cuda, c):
    """Window widths across the sort's digit splits: one radix pass
    (c <= 9), two passes with up to 8 bits each (c <= 17) and wider second
    passes (c = 18, 20)."""
    n = 2777
    sc = wl.make_scalars(n, seed=100 + c)
    logs = wl.make_base_logs(n, seed=200 + c)
    pts = make_bases(logs, 1, cuda)
    assert oracle.same_point(device_msm(pts, sc, 1, cuda, c=c),
                             oracle.generator_multiple(wl.expected_log(sc, logs)))


def test_edge_cases(cuda):
    import torch
    g = oracle.g1_generator()
    # n == 0 -> infinity
    empty = torch.zeros((0, gm.G1_WORDS), dtype=torch.int64, device=cuda)
    out = gm.msm_device(empty, torch.zeros((0, 5), dtype=torch.int64, device=cuda), group=1)
    torch.cuda.synchronize()
    assert not out.any()
    # all-zero scalars
    logs = wl.make_base_logs(50, seed=3)
    pts = make_bases(logs, 1, cuda)
    assert device_msm(pts, np.zeros((50, 5), np.uint64), 1, cuda)[0]["infinity"]
    # infinity bases mixed in: only finite ones count
    host = gm.to_numpy_points(pts, 1).copy()
    host["infinity"][::3] = 1
    sc = wl.make_scalars(50, seed=4)
    got = device_msm(t_dev(host, cuda).reshape(50, -1), sc, 1, cuda)
    assert oracle.same_point(got, oracle.msm_pippenger(host, sc))
    # all bases equal (doubling inside buckets) with scalars 1..N, every c
    N = 64
    pts_eq = t_dev(np.repeat(g, N), cuda).reshape(N, -1)
    sc_eq = np.arange(1, N + 1, dtype=np.uint64).reshape(N, 1)
    for c in (2, 4, 7):
        assert oracle.same_point(device_msm(pts_eq, sc_eq, 1, cuda, c=c), oracle.scalar_mul(g, N * (N + 1) // 2))
    # P and -P with equal scalars cancel; r-1 and full-width scalars
    t = wl.make_base_logs(4, seed=9)
    t[1] = wl.int_to_limbs(pyref.R_ORDER - wl.limbs_to_ints(t[:1])[0])
    k = wl.make_scalars(4, seed=10)
    k[1] = k[0]
    k[2] = wl.int_to_limbs(pyref.R_ORDER - 1)
    k[3] = np.uint64(2 ** 64 - 1)
    pts = make_bases(t, 1, cuda)
    want = oracle.msm_naive(gm.to_numpy_points(pts, 1), k)
    assert oracle.same_point(device_msm(pts, k, 1, cuda), want)


def test_bench_workload_prefix_and_subsets_g1(cuda):
    """The G1 2^20 workload: 2^12 prefix against the reference-structured host
    Pippenger, and 64 random 16-point sub-MSMs against naive double-and-add."""
    n = 1 << 12
    sc = wl.make_scalars(1 << 20, seed=42)[:n]
    logs = wl.make_base_logs(1 << 20, seed=4242)[:n]
    pts = make_bases(logs, 1, cuda)
    check_bases_sample(pts, logs, 1)
    got = device_msm(pts, sc, 1, cuda)
    host = gm.to_numpy_points(pts, 1)
    ref = oracle.ref_msm_pippenger(host, sc, group=1)
    want = ref[0] if ref is not None else oracle.msm_pippenger(host, sc, group=1)
    assert oracle.same_point(got, want)
    rng = np.random.default_rng(64)
    for _ in range(64):
        idx = rng.choice(n, size=16, replace=False)
        sub_pts, sub_sc = host[idx], sc[idx]
        got = device_msm(t_dev(sub_pts, cuda).reshape(16, -1), sub_sc, 1, cuda)
        assert oracle.same_point(got, oracle.msm_naive(sub_pts, sub_sc))


def test_g2_prefix(cuda):
    n = 1 << 10
    sc = wl.make_scalars(1 << 18, seed=43, one_frac=0.0)[:n]
    logs = wl.make_base_logs(1 << 18, seed=4343)[:n]
    pts = make_bases(logs, 2, cuda)
    check_bases_sample(pts, logs, 2, k=4)
    got = device_msm(pts, sc, 2, cuda)
    host = gm.to_numpy_points(pts, 2)
    ref = oracle.ref_msm_pippenger(host, sc, group=2)
    want = ref[0] if ref is not None else oracle.msm_pippenger(host, sc, group=2)
    assert oracle.same_point(got, want)


@pytest.mark.parametrize("group,log2n,seed", [(1, 20, 42), (2, 18, 43)])
def test_full_size_exact_relation(cuda, group, log2n, seed):
    n = 1 << log2n
    sc = wl.make_scalars(n, seed=seed, one_frac=0.01 if group == 1 else 0.0)
    logs = wl.make_base_logs(n, seed=seed * 101)
    pts = make_bases(logs, group, cuda)
    check_bases_sample(pts, logs, group, k=4)
    got = device_msm(pts, sc, group, cuda)
    want = oracle.generator_multiple(wl.expected_log(sc, logs), group=group)
    assert oracle.same_point(got, want)
    # run-to-run: same canonical point on a second call
    assert oracle.same_point(device_msm(pts, sc, group, cuda), got)


def test_concurrent_streams(cuda):
    import torch
    outs, wants = [], []
    streams = [torch.cuda.Stream() for _ in range(3)]
    inputs = []
    for i in range(3):
        n = 2000 + 500 * i
        sc = wl.make_scalars(n, seed=500 + i)
        logs = wl.make_base_logs(n, seed=600 + i)
        inputs.append((make_bases(logs, 1, cuda), t_dev(sc, cuda).reshape(n, -1)))
        wants.append(oracle.generator_multiple(wl.expected_log(sc, logs)))
    for (pts, sc), s in zip(inputs, streams):
        with torch.cuda.stream(s):
            outs.append(gm.msm_device(pts, sc, group=1, stream=s))
    torch.cuda.synchronize()
    for o, w in zip(outs, wants):
        assert oracle.same_point(oracle.proj_to_affine(gm.to_numpy_proj(o, 1), 1), w)


@pytest.mark.parametrize("group,log2n", [(1, 16), (2, 14)])
def test_round_robin_streams(cuda, group, log2n):
    """Consecutive MSMs round-robin over three streams, two per stream (the
    way bench.py times them): one call's reduction tail and host combine run
    while the next calls sort and accumulate, each call on its own pool
    workspace and host-tail slot.  Every result must be its own MSM's."""
    import torch
    n = 1 << log2n
    streams = [torch.cuda.Stream() for _ in range(3)]
    inputs, wants, outs = [], [], []
    for i in range(6):
        sc = wl.make_scalars(n, seed=900 + 10 * group + i)
        logs = wl.make_base_logs(n, seed=950 + 10 * group + i)
        inputs.append((make_bases(logs, group, cuda), t_dev(sc, cuda).reshape(n, -1)))
        wants.append(oracle.generator_multiple(wl.expected_log(sc, logs), group=group))
    torch.cuda.synchronize()
    for i, (pts, sc) in enumerate(inputs):
        s = streams[i % 3]
        with torch.cuda.stream(s):
            outs.append(gm.msm_device(pts, sc, group=group, stream=s))
    torch.cuda.synchronize()
    for o, w in zip(outs, wants):
        assert oracle.same_point(oracle.proj_to_affine(gm.to_numpy_proj(o, group), group), w)


@pytest.mark.parametrize("group,n,c", [(1, 3000, 0), (1, 3000, 8), (1, 5000, 3), (2, 1000, 0)])
def test_heavy_buckets(cuda, group, n, c):
    """Most scalars equal to 1 or 2: a few buckets hold thousands of entries
    and span many accumulation slices (the long-run fix-up path)."""
    rng = np.random.default_rng(n + c)
    sc = wl.make_scalars(n, seed=n + 7 * c + group)
    pick = rng.random(n)
    sc[pick < 0.6] = 0
    sc[pick < 0.6, 0] = 1
    sc[(pick >= 0.6) & (pick < 0.8)] = 0
    sc[(pick >= 0.6) & (pick < 0.8), 0] = 2
    logs = wl.make_base_logs(n, seed=n + 11 * c + group)
    pts = make_bases(logs, group, cuda)
    want = oracle.generator_multiple(wl.expected_log(sc, logs), group=group)
    assert oracle.same_point(device_msm(pts, sc, group, cuda, c=c), want)


def test_plain_msm_graph_capture(cuda):
    """A plain MSM captured into a CUDA graph (device-side window combination)
    and replayed with new scalars."""
    import torch
    n = 3000
    logs = wl.make_base_logs(n, seed=77)
    pts = make_bases(logs, 1, cuda)
    sc0 = wl.make_scalars(n, seed=78)
    static_sc = t_dev(sc0, cuda).reshape(n, -1).clone()
    out = torch.zeros((1, gm.G1P_WORDS), dtype=torch.int64, device=cuda)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        gm.msm_device(pts, static_sc, group=1, out=out, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        gm.msm_device(pts, static_sc, group=1, out=out)
    for seed in (79, 80):
        sc = wl.make_scalars(n, seed=seed)
        static_sc.copy_(t_dev(sc, cuda).reshape(n, -1))
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        got = oracle.proj_to_affine(gm.to_numpy_proj(out, 1), 1)
        assert oracle.same_point(got, oracle.generator_multiple(wl.expected_log(sc, logs)))
    del g


@pytest.mark.parametrize("group", [1, 2])
def test_host_async_two_streams(cuda, group):
    """gm_g{1,2}_msm_host_async: several host-buffer MSMs in flight on two
    streams (pinned buffers), each result equal to the exact relation; the
    empty MSM gives the identity; bad arguments are rejected."""
    import torch
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    adt, pdt = (gm.G1, gm.G1P) if group == 1 else (gm.G2, gm.G2P)
    words = gm.G1_WORDS if group == 1 else gm.G2_WORDS
    pwords = gm.G1P_WORDS if group == 1 else gm.G2P_WORDS
    cases = []
    for i, n in enumerate((700, 3000, 1, 2500)):
        logs = wl.make_base_logs(n, seed=800 + i + 10 * group)
        sc = wl.make_scalars(n, seed=900 + i + 10 * group)
        pts = make_bases(logs, group, cuda)
        pts_pin = torch.empty((n, words), dtype=torch.int64, pin_memory=True)
        pts_pin.copy_(pts.cpu())
        sc_pin = torch.empty((n, 5), dtype=torch.int64, pin_memory=True)
        sc_pin.copy_(torch.from_numpy(sc.view(np.int64)))
        cases.append((pts_pin, sc_pin, oracle.generator_multiple(wl.expected_log(sc, logs), group=group)))
    res = torch.zeros((len(cases) + 1, pwords), dtype=torch.int64, pin_memory=True)
    err = torch.ones(len(cases) + 1, dtype=torch.int32, pin_memory=True)
    res_np = res.numpy().view(np.uint64).view(pdt).reshape(-1)
    err_np = err.numpy().view(np.uint32)
    for i, (pts_pin, sc_pin, _) in enumerate(cases):
        gm.msm_host_async(pts_pin.numpy().view(np.uint64).view(adt).reshape(-1), sc_pin.numpy().view(np.uint64),
                          res_np[i:i + 1], group=group, stream=streams[i % 2], err=err_np[i:i + 1])
    empty = np.zeros(0, dtype=adt)
    k = len(cases)
    res_np[k]["X"] = 5  # must be overwritten with the identity
    gm.msm_host_async(empty, np.zeros((0, 5), dtype=np.uint64), res_np[k:k + 1], group=group, stream=streams[0],
                      err=err_np[k:k + 1])
    for s in streams:
        s.synchronize()
    assert err_np.max() == 0
    for i, (_, _, want) in enumerate(cases):
        assert oracle.same_point(oracle.proj_to_affine(res_np[i:i + 1], group), want), i
    assert oracle.proj_to_affine(res_np[k:k + 1], group)[0]["infinity"]
    L = gm.lib()
    fn = L.gm_g1_msm_host_async if group == 1 else L.gm_g2_msm_host_async
    assert fn(None, 0, None, None, None, 5, 10, 1, None) == -1
    assert fn(None, 0, res_np[:1].ctypes.data, res_np[:1].ctypes.data, res_np[:1].ctypes.data, 9, 1, 1, None) == -1


@pytest.mark.parametrize("group,n", [(1, (1 << 24) - 3), (2, (1 << 21) + 5)])
def test_max_size_exact_relation(cuda, group, n):
    """Well past the benchmark sizes, with ragged n: 2^24 - 3 G1 points and
    2^21 + 5 G2 points against the exact relation sum k_i t_i (mod r), and
    linearity: the MSM of the whole equals the sum of the MSMs of two
    unequal parts."""
    import torch
    sc = wl.make_scalars(n, seed=7000 + group)
    logs = wl.make_base_logs(n, seed=7100 + group)
    pts = make_bases(logs, group, cuda)
    sc_t = t_dev(sc, cuda).reshape(n, -1)
    got = device_msm(pts, sc_t, group, cuda)
    want = oracle.generator_multiple(wl.expected_log(sc, logs), group=group)
    assert oracle.same_point(got, want)
    cut = n // 3
    a = gm.msm_device(pts[:cut].contiguous(), sc_t[:cut].contiguous(), group=group)
    b = gm.msm_device(pts[cut:].contiguous(), sc_t[cut:].contiguous(), group=group)
    both = torch.stack([a, b])
    s = gm.sum_projective(both, group=group)
    torch.cuda.synchronize()
    assert oracle.same_point(oracle.proj_to_affine(gm.to_numpy_proj(s, group), group), want)


@pytest.mark.parametrize("group,log2n,c", [(1, 16, 0), (1, 12, 5), (2, 14, 0)])
def test_projective_output_is_deterministic(cuda, group, log2n, c):
    """The sort orders every bucket's entries by point index (no atomics
    decide an order), so repeated MSMs on the same inputs give the same
    projective coordinates word for word, not only the same point; also
    across streams and with a busy GPU in between."""
    import torch
    n = 1 << log2n
    sc = t_dev(wl.make_scalars(n, seed=1300 + log2n), cuda).reshape(n, -1)
    pts = make_bases(wl.make_base_logs(n, seed=1400 + log2n), group, cuda)
    first = gm.msm_device(pts, sc, group=group, window_bits=c).clone()
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in range(2)]
    outs = []
    for i in range(4):
        s = streams[i % 2]
        with torch.cuda.stream(s):
            outs.append(gm.msm_device(pts, sc, group=group, window_bits=c, stream=s))
    torch.cuda.synchronize()
    for o in outs:
        assert torch.equal(o, first)
