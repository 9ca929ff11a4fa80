"""CPU: the field constants compiled into the CUDA kernels.

The constants are parsed from gpu_msm_b200/csrc/field.cuh and checked against
the modulus of the workload module (the reference's p, src/fp.cu:15): p, 2p,
R^2 mod p, R mod p and -p^-1 mod 2^32 (R = 2^448), and the bound 4p < R that
lets product operands stay below 2p.
"""
import os
import re

from gpu_msm_b200.workload import P_MODULUS as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
R = 1 << 448


def _const(name):
    src = open(os.path.join(ROOT, "gpu_msm_b200", "csrc", "field.cuh")).read()
    m = re.search(r"static constexpr uint32_t %s\(int i\) \{(.*?)default" % name, src, re.S)
    assert m, name
    words = {int(k): int(v, 16) for k, v in re.findall(r"case (\d+): return 0x([0-9a-f]+)u;", m.group(1))}
    return sum(v << (32 * k) for k, v in words.items())


def test_constants_match_the_modulus():
    assert _const("P") == P
    assert _const("P2") == 2 * P
    assert _const("R2") == R * R % P
    assert _const("ONE") == R % P
    assert 4 * P < R
    src = open(os.path.join(ROOT, "gpu_msm_b200", "csrc", "field.cuh")).read()
    pinv = int(re.search(r"PINV = 0x([0-9a-f]+)u", src).group(1), 16)
    assert (pinv * P) % (1 << 32) == (1 << 32) - 1
