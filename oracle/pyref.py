"""Pure-Python big-integer restatement of the BLS12-446 arithmetic.

TEST INFRASTRUCTURE ONLY.  Values here are plain integers in standard form
(not Montgomery).  It is the third, independent check beside the C
restatement (oracle.c) and the reference host code (_ref/libref.so), and it
generates the golden fixtures under tests/golden/.

Constants follow pdroalves/gpu_msm src/fp.cu:15-33 (p, R = 2^448) and the
generators of src/curve.cu:786-814.  The scalar-field order r is not in the
reference: it is derived from the BLS12 parameter u (p = (u-1)^2 (u^4-u^2+1)/3
+ u, r = u^4 - u^2 + 1); tests/test_oracle.py checks r*G = O on both groups.
"""
from __future__ import annotations

P = 0x3CDEE0FB28C5E535200FC34965AAD6400095A4B78A02FE320F75A64BBAC71602824E6DC3E23ACDEE56EE4528C573B5CC311C0026AAB0AAAB
R_MONT = 1 << 448
U_PARAM = -0x6008204000000020001
R_ORDER = U_PARAM ** 4 - U_PARAM ** 2 + 1

assert (U_PARAM - 1) ** 2 * R_ORDER // 3 + U_PARAM == P

G1_X = 0x326ED6BD777FC6A311B73D3D76AE98512CE8C34265BF38416B20D782901A6F6211C1E56B3E4BC80B8BC02B7CBE6A9E8D3BF9166C8236F4FA
G1_Y = 0x1A7CAF4A4D3887A6D6D62D244E413636F843C947AA57F57139D7F424B6660204B9093F32002756DA22DB0CE6034A9DB9FE6F792612016B30
G2_X = (0x21F8D4A76F74541AA57C0038441F7D1518DAD8ED784DD225062B61439640E885043C6BF16312D638D6EBAF149094F1CC0E529EE4DCE9991D,
        0x1E0F563C601BB8DCA1B4E791D1B86560DEBAF4A2C553452771449CDECA4F00072879DD439B019B8B7CEF6ACB145B6413CAF5185423A7D23A)
G2_Y = (0x115EA2305A78F6460CC61570301497A7DDFF621B5DB3F8970177BFD6654E681E00346CEBAD16A03682039E4221FF3507274315837455B919,
        0x25ED2192B203C1FE76A2FFCB7D47679D0B0BCC3FB6F2161C7532834528CD5A648A8E6755F9D82FD1D8AB17C84B9F03CD392236E9CF2976C2)

B_G1 = 1            # y^2 = x^3 + 1   (what the generator satisfies)
B_G2 = (1, 1)       # y^2 = x^3 + (1 + i)


def to_mont(v: int) -> int:
    return v * R_MONT % P


def from_mont(v: int) -> int:
    return v * pow(R_MONT, -1, P) % P


# ---- Fp2 = Fp[i]/(i^2 + 1) -------------------------------------------------

def f2_add(a, b):
    return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)


def f2_sub(a, b):
    return ((a[0] - b[0]) % P, (a[1] - b[1]) % P)


def f2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def f2_inv(a):
    n = (a[0] * a[0] + a[1] * a[1]) % P
    ni = pow(n, -1, P)
    return (a[0] * ni % P, (-a[1]) * ni % P)


class Fp1:
    """Field ops for G1 (plain ints)."""
    zero = 0
    one = 1

    @staticmethod
    def add(a, b): return (a + b) % P
    @staticmethod
    def sub(a, b): return (a - b) % P
    @staticmethod
    def mul(a, b): return a * b % P
    @staticmethod
    def inv(a): return pow(a, -1, P)
    @staticmethod
    def neg(a): return (-a) % P
    @staticmethod
    def small(k): return k % P


class Fp2F:
    """Field ops for G2 (pairs)."""
    zero = (0, 0)
    one = (1, 0)
    add = staticmethod(f2_add)
    sub = staticmethod(f2_sub)
    mul = staticmethod(f2_mul)
    inv = staticmethod(f2_inv)

    @staticmethod
    def neg(a): return ((-a[0]) % P, (-a[1]) % P)
    @staticmethod
    def small(k): return (k % P, 0)


def _field(group):
    return Fp1 if group == 1 else Fp2F


def add(p, q, group=1):
    """Affine addition; None is the point at infinity."""
    F = _field(group)
    if p is None:
        return q
    if q is None:
        return p
    x1, y1 = p
    x2, y2 = q
    if x1 == x2:
        if y1 == F.neg(y2):
            return None
        lam = F.mul(F.mul(F.small(3), F.mul(x1, x1)), F.inv(F.add(y1, y1)))
    else:
        lam = F.mul(F.sub(y2, y1), F.inv(F.sub(x2, x1)))
    x3 = F.sub(F.sub(F.mul(lam, lam), x1), x2)
    y3 = F.sub(F.mul(lam, F.sub(x1, x3)), y1)
    return (x3, y3)


def mul(p, k: int, group=1):
    acc = None
    base = p
    while k > 0:
        if k & 1:
            acc = add(acc, base, group)
        base = add(base, base, group)
        k >>= 1
    return acc


def msm(points, scalars, group=1):
    acc = None
    for p, k in zip(points, scalars):
        acc = add(acc, mul(p, k, group), group)
    return acc


def g1():
    return (G1_X, G1_Y)


def g2():
    return (G2_X, G2_Y)


def on_curve(p, group=1) -> bool:
    if p is None:
        return True
    F = _field(group)
    x, y = p
    b = B_G1 if group == 1 else B_G2
    return F.mul(y, y) == F.add(F.mul(F.mul(x, x), x), b)
