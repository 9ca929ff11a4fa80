"""Generate tests/golden/arkworks_limbs.json: BLS12-446 points and scalars in
the two limb forms an arkworks / tfhe-zk-pok caller can hand over (run from
the repo root: ``python tests/golden/make_arkworks_fixture.py``).

The reference's Rust crate marshals tfhe-zk-pok points into its C structs
(pdroalves/gpu_msm rust-api/src/conversions.rs:56-79, types.rs:345-376,
:492-533) through ``PrimeField::into_bigint()``, which in ark-ff returns the
canonical integer of a field element ("normal form"; the crate's own G1 test,
rust-api/src/example.rs:161-163, relies on that).  ark-ff's Montgomery
backend stores every element internally as x * R mod p with R = 2^(64 N) for
N 64-bit limbs: for the 446-bit prime, N = 7 and R = 2^448, the Montgomery
radix of this library.  So the two hand-offs are
* ``into_bigint()`` limbs  -> ``points_montgomery = 0`` (converted on the device);
* the raw internal limbs  -> ``points_montgomery = 1`` (used unchanged);
and a scalar-field element's ``into_bigint()`` (r is 299 bits, N = 5 limbs)
is a 5-limb scalar row.

Points are k * G from the pure-Python big-integer restatement of the curve
(oracle/pyref.py); the expected MSM is given in both forms too.
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
RM = 1 << 448


def limbs(v: int, n: int = 7):
    return [hex((v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF) for i in range(n)]


def coord(v, group, mont: bool):
    if group == 1:
        return limbs(v * RM % P if mont else v)
    return [limbs(c * RM % P if mont else c) for c in v]


def point(pt, group, mont: bool):
    if pt is None:
        return {"infinity": True}
    return {"infinity": False, "x": coord(pt[0], group, mont), "y": coord(pt[1], group, mont)}


def case(group, n, seed):
    rng = random.Random(seed)
    gen = pyref.g1() if group == 1 else pyref.g2()
    ks = [rng.randrange(1, pyref.R_ORDER) for _ in range(n)]
    pts = [pyref.mul(gen, k, group) for k in ks]
    scalars = [rng.randrange(pyref.R_ORDER) for _ in range(n)]
    scalars[0] = 1
    if n > 2:
        scalars[1] = 0
    want = pyref.msm(pts, scalars, group)
    return {
        "group": group,
        "into_bigint_points": [point(p, group, False) for p in pts],
        "internal_points": [point(p, group, True) for p in pts],
        "scalars": [limbs(s, 5) for s in scalars],
        "msm_into_bigint": point(want, group, False),
        "msm_internal": point(want, group, True),
    }


def main():
    out = {
        "doc": "into_bigint = canonical limbs; internal = x * 2^448 mod p (ark-ff Montgomery, 7 limbs); "
               "scalars = Fr into_bigint (5 limbs)",
        "cases": [case(1, 9, 446), case(2, 5, 447)],
    }
    path = os.path.join(HERE, "arkworks_limbs.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
