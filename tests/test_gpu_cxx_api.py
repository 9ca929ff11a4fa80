"""GPU: the reference-compatible C++ API (include/gpu_msm_b200_cxx.h).

tests/cxx/cxx_api_driver is compiled against that header and linked with
libgpu_msm_b200.so; it calls point_msm_u64_g1/_g2, point_msm<G1Point|G2Point>
(affine result), point_to_montgomery_batch, fp_{mul,add}_array_{host,device}
and fp2_{mul,add}_array_host the way a caller of the reference's curve.h /
fp_kernels.h / fp2_kernels.h does.  Every output is checked against the
oracle, bit-exact (points in canonical affine form).
"""
import os
import random
import subprocess

import numpy as np
import pytest

import gpu_msm_b200 as gm
import oracle
from gpu_msm_b200 import workload as wl
from oracle import pyref

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "cxx", "_build", "cxx_api_driver")


def _driver():
    if not os.path.exists(DRIVER):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "tests", "cxx")])
    return DRIVER


def _group_inputs(d, group, n, seed, cuda):
    import torch
    logs = wl.make_base_logs(n, seed=seed)
    pts_t = gm.generator_mul_batch(torch.from_numpy(logs.view(np.int64)).to(cuda), group=group)
    torch.cuda.synchronize()
    pts = gm.to_numpy_points(pts_t, group)
    k5 = wl.make_scalars(n, seed=seed + 1)
    rng = np.random.default_rng(seed + 2)
    k64 = rng.integers(0, 2 ** 64, size=(n, 1), dtype=np.uint64)
    k64[::17] = 0
    tag = f"g{group}"
    pts.tofile(os.path.join(d, f"in_{tag}_points.bin"))
    k64.tofile(os.path.join(d, f"in_{tag}_scalars_u64.bin"))
    k5.tofile(os.path.join(d, f"in_{tag}_scalars_5.bin"))
    oracle.from_mont(pts[:32], group).tofile(os.path.join(d, f"in_{tag}_points_std.bin"))
    return pts, logs, k64, k5


def test_cxx_api_matches_oracle(cuda, tmp_path):
    d = str(tmp_path)
    groups = {1: _group_inputs(d, 1, 300, 901, cuda), 2: _group_inputs(d, 2, 64, 902, cuda)}
    rnd = random.Random(903)
    P = pyref.P
    xs = [rnd.randrange(P) for _ in range(200)] + [0, 1, P - 1, P - 1]
    ys = [rnd.randrange(P) for _ in range(200)] + [P - 1, P - 1, 1, P - 1]
    a, b = oracle.ints_to_fp_array(xs), oracle.ints_to_fp_array(ys)
    a.tofile(os.path.join(d, "in_fp_a.bin"))
    b.tofile(os.path.join(d, "in_fp_b.bin"))
    a2 = np.stack([a[:100], a[100:200]], axis=1)
    b2 = np.stack([b[:100], b[100:200]], axis=1)
    a2.tofile(os.path.join(d, "in_fp2_a.bin"))
    b2.tofile(os.path.join(d, "in_fp2_b.bin"))

    out = subprocess.run([_driver(), d], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr

    def rd(name, dtype):
        return np.fromfile(os.path.join(d, name), dtype=dtype)

    for group, (pts, logs, k64, k5) in groups.items():
        tag = f"g{group}"
        pdt = gm.G1P if group == 1 else gm.G2P
        adt = gm.G1 if group == 1 else gm.G2
        prj = rd(f"out_{tag}_msm_u64.bin", pdt)
        assert oracle.same_point(oracle.proj_to_affine(prj[:1], group),
                                 oracle.generator_multiple(wl.expected_log(k64, logs), group=group))
        assert oracle.proj_to_affine(prj[1:2], group)[0]["infinity"]
        aff = rd(f"out_{tag}_msm_affine.bin", adt)
        assert oracle.same_point(aff[:1], oracle.generator_multiple(wl.expected_log(k5, logs), group=group))
        assert aff[1]["infinity"]
        conv = rd(f"out_{tag}_to_mont.bin", adt)
        assert oracle.same_point(conv, pts[:32])

    assert np.array_equal(rd("out_fp_mul_host.bin", np.uint64).reshape(a.shape), oracle.fp_mul(a, b))
    assert np.array_equal(rd("out_fp_mul_device.bin", np.uint64).reshape(a.shape), oracle.fp_mul(a, b))
    want_add = oracle.ints_to_fp_array([(x + y) % P for x, y in zip(xs, ys)])
    assert np.array_equal(rd("out_fp_add_host.bin", np.uint64).reshape(a.shape), want_add)
    assert np.array_equal(rd("out_fp_add_device.bin", np.uint64).reshape(a.shape), want_add)
    assert np.array_equal(rd("out_fp2_mul_host.bin", np.uint64).reshape(a2.shape), oracle.fp2_mul(a2, b2))
    want2 = np.stack([want_add[:100], want_add[100:200]], axis=1)
    assert np.array_equal(rd("out_fp2_add_host.bin", np.uint64).reshape(a2.shape), want2)

    # single-element stream APIs and host-pointer helpers (fp.h:158-204,
    # fp2.h:99-133, curve.h:156-205, fp_kernels.h:26-38, fp2_kernels.h:21-37)
    from tests import element_cases as ec
    x, y = xs[0], ys[0]
    fe = lambda op, a=0, b=0, c=0, arg=0: pyref.fp_elem(op, a, b, c, arg)[0]  # noqa: E731
    want_fp = [fe("add", x, y), fe("sub", x, y), fe("mul", x, y), fe("div", x, y), fe("mont_mul", x, y),
               fe("neg", x), fe("inv", x), fe("to_mont", x), fe("from_mont", x), x, 0, 1,
               fe("add", x, y), fe("sub", x, y), fe("mul", x, y), fe("neg", x), fe("inv", x), fe("div", x, y),
               fe("to_mont", x), fe("from_mont", x), fe("mont_mul", x, y), x, x, y, fe("pow_u64", x, arg=65537),
               fe("sqrt", x * x % P)]
    got_fp = rd("out_elem_fp.bin", np.uint64).reshape(-1, 7)
    assert [ec.fp_int(r) for r in got_fp] == want_fp
    x2, y2 = (xs[0], xs[100]), (ys[0], ys[100])
    f2 = lambda op, a, b=(0, 0): pyref.fp2_elem(op, a, b)[0]  # noqa: E731
    want_fp2 = [f2("add", x2, y2), f2("sub", x2, y2), f2("mul", x2, y2), f2("div", x2, y2), f2("square", x2),
                f2("neg", x2), f2("conjugate", x2), f2("inv", x2), x2,
                f2("add", x2, y2), f2("sub", x2, y2), f2("mul", x2, y2), f2("neg", x2), f2("conjugate", x2),
                f2("square", x2), f2("inv", x2), f2("div", x2, y2), f2("mul_by_i", x2), f2("frobenius", x2), x2,
                x2]
    got_fp2 = rd("out_elem_fp2.bin", np.uint64).reshape(-1, 14)
    assert [ec.fp2_int(r) for r in got_fp2] == want_fp2
    want_flags = [1, pyref.fp_elem("cmp", x, y)[1], int(x == 0), 1, pyref.fp_elem("is_qr", x)[1],
                  pyref.fp2_elem("cmp", x2, y2)[1], 0, 0]
    assert rd("out_elem_flags.bin", np.int32).tolist() == want_flags
    for group, (pts, logs, k64, k5) in groups.items():
        p0, p1 = ec.point_from_np(pts[0:1], group), ec.point_from_np(pts[1:2], group)
        k5i = oracle.limbs_to_int(k5[0])
        std0 = ec.point_from_np(oracle.from_mont(pts[:1], group), group)
        want = [ec.expected_point("add", p0, p1, 0, 0, group), ec.expected_point("double", p0, None, 0, 0, group),
                ec.expected_point("neg", p0, None, 0, 0, group),
                ec.expected_point("scalar_mul_u64", p0, None, int(k64[0, 0]), 0, group),
                ec.expected_point("scalar_mul", p0, None, k5i, 5, group),
                ec.expected_point("to_mont", std0, None, 0, 0, group),
                ec.expected_point("from_mont", p0, None, 0, 0, group)]
        got = rd(f"out_elem_g{group}.bin", gm.G1 if group == 1 else gm.G2)
        assert [ec.point_from_np(got[i:i + 1], group) for i in range(7)] == want, group
