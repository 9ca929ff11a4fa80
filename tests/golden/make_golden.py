"""Generates the golden fixtures in tests/golden/ (run from the repo root:
``python tests/golden/make_golden.py``).

Sources:
* ``field_kat.json`` -- the known-answer vectors of the reference's own tests
  (pdroalves/gpu_msm tests/test_fp.cu, tests/test_fp2.cu), restated as
  (inputs, expected) pairs, plus seeded random pairs whose expected products
  come from the pure-Python big-integer restatement (oracle/pyref.py).
* ``msm_golden.json`` -- MSM cases: the reference's relation tests
  sum_{i=1..N} i*G = N(N+1)/2 * G (tests/test_msm.cu:132-592) for G1 N=10,
  N=100 and G2 N=10, and seeded random MSMs (random bases k*G, scalars in
  [0, r) with zeros, ones, duplicates and a negated pair), all with expected
  canonical affine outputs in standard form from oracle/pyref.py.
When the reference host code was built (oracle/_ref/libref.so), every MSM
fixture is also recomputed by the reference's own host functions and must
agree; the script aborts otherwise.
"""
from __future__ import annotations

import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyref  # noqa: E402

P = pyref.P
R = pyref.R_ORDER
RM = 1 << 448


def hx(v: int) -> str:
    return hex(v)


def fp2_hex(v):
    return [hx(v[0]), hx(v[1])]


def point_json(pt, group):
    if pt is None:
        return {"infinity": True}
    if group == 1:
        return {"infinity": False, "x": hx(pt[0]), "y": hx(pt[1])}
    return {"infinity": False, "x": fp2_hex(pt[0]), "y": fp2_hex(pt[1])}


def field_kats():
    kats = []
    # tests/test_fp.cu:1062 (p-1)*(p-1) = 1 (normal-form fp_mul)
    kats.append({"op": "fp_mul", "a": hx(P - 1), "b": hx(P - 1), "c": hx(1), "src": "tests/test_fp.cu:1062"})
    # tests/test_fp.cu:999 50 - 100 = p - 50
    kats.append({"op": "fp_sub", "a": hx(50), "b": hx(100), "c": hx(P - 50), "src": "tests/test_fp.cu:999"})
    # tests/test_fp.cu:1146 (p-1) + 1 = 0
    kats.append({"op": "fp_add", "a": hx(P - 1), "b": hx(1), "c": hx(0), "src": "tests/test_fp.cu:1146"})
    # tests/test_fp.cu:1088 a*2 = a+a
    limbs = [0x18e00013555855, 0x2b772294629DAE6, 0x412736E1F11D66F7, 0x7BAD325DD638B01, 0x4CAD5BC5017F19,
             0x1007E1A4B2D56B20, 0x1E6F707D9462F2]
    a = sum(v << (64 * i) for i, v in enumerate(limbs))
    kats.append({"op": "fp_mul", "a": hx(a), "b": hx(2), "c": hx(2 * a % P), "src": "tests/test_fp.cu:1088"})
    # tests/test_fp.cu:1025 2^200 * 2^100 = 2^300
    kats.append({"op": "fp_mul", "a": hx(1 << 200), "b": hx(1 << 100), "c": hx((1 << 300) % P),
                 "src": "tests/test_fp.cu:1025"})
    # tests/test_fp2.cu:196 (1+i)^2 = 2i ; tests/test_fp2.cu:222 i*i = -1
    kats.append({"op": "fp2_mul", "a": [hx(1), hx(1)], "b": [hx(1), hx(1)], "c": [hx(0), hx(2)],
                 "src": "tests/test_fp2.cu:196"})
    kats.append({"op": "fp2_mul", "a": [hx(0), hx(1)], "b": [hx(0), hx(1)], "c": [hx(P - 1), hx(0)],
                 "src": "tests/test_fp2.cu:222"})
    # Montgomery-form products on random canonical inputs
    rng = random.Random(42)
    for _ in range(64):
        x, y = rng.randrange(P), rng.randrange(P)
        kats.append({"op": "fp_mont_mul", "a": hx(x), "b": hx(y), "c": hx(x * y * pow(RM, -1, P) % P),
                     "src": "pyref"})
    edge = [0, 1, P - 1, P - 2, (1 << 445), P >> 1, (1 << 448) % P]
    for x in edge:
        for y in edge:
            kats.append({"op": "fp_mont_mul", "a": hx(x), "b": hx(y), "c": hx(x * y * pow(RM, -1, P) % P),
                         "src": "pyref edge"})
    for _ in range(32):
        a = (rng.randrange(P), rng.randrange(P))
        b = (rng.randrange(P), rng.randrange(P))
        am = tuple(v * RM % P for v in a)
        bm = tuple(v * RM % P for v in b)
        cm = pyref.f2_mul(pyref.f2_mul(am, bm), (pow(RM, -1, P), 0))
        kats.append({"op": "fp2_mont_mul", "a": fp2_hex(am), "b": fp2_hex(bm), "c": fp2_hex(cm), "src": "pyref"})
    return kats


def msm_cases():
    cases = []
    g1, g2 = pyref.g1(), pyref.g2()
    # relation tests of tests/test_msm.cu
    for group, gen, N, src in ((1, g1, 10, "tests/test_msm.cu:132"), (2, g2, 10, "tests/test_msm.cu:366"),
                               (1, g1, 100, "tests/test_msm.cu:487")):
        cases.append({
            "name": f"relation_g{group}_N{N}", "group": group, "src": src, "limbs": 1,
            "bases_k": [1] * N, "scalars": [hx(i + 1) for i in range(N)],
            "expected": point_json(pyref.mul(gen, N * (N + 1) // 2, group), group)})
    rng = random.Random(7)
    for group, gen, n in ((1, g1, 33), (2, g2, 17)):
        ks = [rng.randrange(1, R) for _ in range(n)]
        sc = [rng.randrange(R) for _ in range(n)]
        sc[3] = 0
        sc[5] = 1
        ks[7] = ks[2]          # duplicated base
        ks[9] = R - ks[8]      # P_9 = -P_8
        sc[9] = sc[8]          # ... with equal scalars: the pair cancels
        s = sum(k * v for k, v in zip(ks, sc)) % R
        cases.append({
            "name": f"random_g{group}_n{n}", "group": group, "src": "pyref", "limbs": 5,
            "bases_k": [hx(k) for k in ks], "scalars": [hx(v) for v in sc],
            "expected": point_json(pyref.mul(gen, s, group), group)})
    # all scalars zero -> infinity
    cases.append({"name": "zero_scalars_g1", "group": 1, "src": "pyref", "limbs": 5,
                  "bases_k": [hx(3), hx(5)], "scalars": [hx(0), hx(0)], "expected": {"infinity": True}})
    # scalar r-1 on G: -G
    cases.append({"name": "r_minus_1_g1", "group": 1, "src": "pyref", "limbs": 5,
                  "bases_k": [hx(1)], "scalars": [hx(R - 1)],
                  "expected": point_json(pyref.mul(g1, R - 1, 1), 1)})
    return cases


def check_against_reference(cases):
    """Recompute every MSM fixture with the reference host code when built."""
    import numpy as np

    import oracle
    if oracle.ref_lib() is None:
        print("reference host code not built: skipping the cross-check")
        return
    for c in cases:
        g = c["group"]
        gen = oracle.g1_generator() if g == 1 else oracle.g2_generator()
        pts = np.concatenate([oracle.scalar_mul(gen, int(k, 16) if isinstance(k, str) else k, group=g)
                              for k in c["bases_k"]])
        L = c["limbs"]
        sc = np.array([[(int(v, 16) >> (64 * j)) & (2 ** 64 - 1) for j in range(L)] for v in c["scalars"]],
                      dtype=np.uint64)
        aff, _ = oracle.ref_msm_pippenger(pts, sc, group=g)
        std = oracle.from_mont(aff, group=g)[0]
        exp = c["expected"]
        if exp["infinity"]:
            assert std["infinity"], c["name"]
            continue
        if g == 1:
            got = (oracle.limbs_to_int(std["x"]), oracle.limbs_to_int(std["y"]))
            want = (int(exp["x"], 16), int(exp["y"], 16))
        else:
            got = (oracle.limbs_to_int(std["x"][0]), oracle.limbs_to_int(std["x"][1]),
                   oracle.limbs_to_int(std["y"][0]), oracle.limbs_to_int(std["y"][1]))
            want = tuple(int(v, 16) for v in exp["x"] + exp["y"])
        assert got == want, f"reference host code disagrees on {c['name']}"
        print("reference agrees:", c["name"])


def main():
    kats = field_kats()
    cases = msm_cases()
    check_against_reference(cases)
    with open(os.path.join(HERE, "field_kat.json"), "w") as f:
        json.dump({"p": hx(P), "r": hx(R), "kats": kats}, f, indent=1)
    with open(os.path.join(HERE, "msm_golden.json"), "w") as f:
        json.dump({"cases": cases}, f, indent=1)
    print(f"wrote {len(kats)} field KATs and {len(cases)} MSM cases")


if __name__ == "__main__":
    main()
