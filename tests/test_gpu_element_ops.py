"""GPU: the single-element operations behind the reference's stream APIs
(gm_fp_elem, gm_fp2_elem, gm_g{1,2}_point_elem; include/fp.h:158-204,
include/fp2.h:99-133, include/curve.h:156-211), bit-exact against the oracle
(oracle/pyref.py, itself pinned to the reference's host code by
tests/test_element_oracle.py) on every case of tests/element_cases.py:
edge values, inverses of zero, non-residues, the reference's degenerate
affine-add branch, infinity flags with coordinates left in place, full-width
and u64 scalars."""
import numpy as np
import pytest
import torch

import gpu_msm_b200 as gm
from oracle import pyref
from tests import element_cases as ec

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).reshape(1, -1).copy()).to(cuda)


def _run_field(cases, cuda, fp2):
    to_np = ec.fp2_np if fp2 else ec.fp_np
    outs = []
    for op, a, b, c, arg in cases:
        ta, tb, tc = _dev(to_np(a), cuda), _dev(to_np(b), cuda), _dev(to_np(c), cuda)
        outs.append(gm.field_elem(op, ta, tb, tc, arg=arg, fp2=fp2))
    torch.cuda.synchronize()
    return outs


def test_fp_elem_matches_oracle(cuda):
    cases = ec.fp_cases()
    outs = _run_field(cases, cuda, fp2=False)
    for (op, a, b, c, arg), (tc, tf) in zip(cases, outs):
        want, flag = pyref.fp_elem(op, a, b, c, arg)
        got = ec.fp_int(tc.cpu().numpy().view(np.uint64).reshape(-1))
        if want is not None:
            assert got == want, (op, a, b, arg)
        else:
            assert got == c, op  # predicates leave c alone
        if op in ("cmp", "is_zero", "is_one", "is_qr", "sqrt"):
            assert int(tf.item()) == flag, (op, a, b)


def test_fp2_elem_matches_oracle(cuda):
    cases = ec.fp2_cases()
    outs = _run_field(cases, cuda, fp2=True)
    for (op, a, b, c, arg), (tc, tf) in zip(cases, outs):
        want, flag = pyref.fp2_elem(op, a, b, c, arg)
        got = ec.fp2_int(tc.cpu().numpy().view(np.uint64).reshape(-1))
        assert got == (want if want is not None else c), (op, a, b)
        if op in ("cmp", "is_zero", "is_one"):
            assert int(tf.item()) == flag, (op, a, b)


@pytest.mark.parametrize("group", [1, 2])
def test_point_elem_matches_oracle(cuda, group):
    cases = ec.point_cases(group)
    outs = []
    for op, p, q, k, limbs in cases:
        tp = _dev(ec.point_np(p, group).view(np.uint64), cuda) if p is not None else None
        tq = _dev(ec.point_np(q, group).view(np.uint64), cuda) if q is not None else None
        ts = _dev(ec.oracle.int_to_limbs(k, limbs), cuda) if limbs > 0 else None
        out = gm.point_elem(op, tp, tq, scalar=ts, scalar_u64=k if limbs == 0 else 0, group=group)
        outs.append(out)
    torch.cuda.synchronize()
    dt = gm.G1 if group == 1 else gm.G2
    for (op, p, q, k, limbs), out in zip(cases, outs):
        got = ec.point_from_np(out.cpu().numpy().view(np.uint64).view(dt), group)
        assert got == ec.expected_point(op, p, q, k, limbs, group), (op, k, limbs)


def test_elem_rejects_bad_arguments(cuda):
    L = gm.lib()
    assert L.gm_fp_elem(None, 0, 99, None, None, None, 0, None) == -1
    assert L.gm_fp_elem(None, 0, gm.FP_OPS.index("add"), None, None, None, 0, None) == -1
    assert L.gm_fp2_elem(None, 0, gm.FP2_OPS.index("cmp"), None, None, None, 0, None) == -1
    assert L.gm_g1_point_elem(None, 0, 99, None, None, None, None, 0, 0) == -1
    assert L.gm_g2_point_elem(None, 0, gm.POINT_OPS.index("add"), None, None, None, None, 0, 0) == -1


@pytest.mark.parametrize("group", [1, 2])
def test_on_curve_batch(cuda, group):
    """Batched on-curve check with the constants the generators satisfy
    (b = 1, b' = 1 + i): multiples of G pass, infinity passes, points with a
    perturbed coordinate fail; the answers equal the oracle's."""
    from gpu_msm_b200 import workload as wl
    from oracle import pyref as pr
    n = 300
    logs = wl.make_base_logs(n, seed=77 + group)
    pts_t = gm.generator_mul_batch(torch.from_numpy(logs.view(np.int64)).to(cuda), group=group)
    pts = gm.to_numpy_points(pts_t, group).copy()
    bad = np.arange(n) % 3 == 1
    for i in np.nonzero(bad)[0]:  # y += 1 (Montgomery one added to the first limb word set)
        y = ec.point_from_np(pts[i:i + 1], group)
        F = pr._field(group)
        y1 = F.add(y[1], F.small(pr.to_mont(1)) if group == 1 else (pr.to_mont(1), 0))
        pts[i:i + 1] = ec.point_np((y[0], y1, False), group)
    pts["infinity"][::7] = 1
    ok = gm.on_curve(torch.from_numpy(pts.view(np.uint64).view(np.int64).reshape(n, -1)).to(cuda), group=group)
    got = ok.cpu().numpy()
    want = []
    for i in range(n):
        x, y, inf = ec._std_pt(ec.point_from_np(pts[i:i + 1], group), group)
        want.append(1 if inf or pr.on_curve((x, y), group) else 0)
    assert got.tolist() == want
    assert got.sum() < n and got.sum() > n // 2
