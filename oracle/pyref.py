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


# ---- single-element operations (the reference's stream APIs) ----------------
# Standard-form ints in, (result, flag) out, with the conventions of
# src/fp.cu (fp_add ... fp_sqrt), src/fp2.cu and src/curve.cu:72-268.

R_INV = pow(R_MONT, -1, P)


def _inv0(v):
    return pow(v, P - 2, P)  # Fermat: 0 -> 0 like fp_inv (src/fp.cu:522)


def fp_elem(op, a=0, b=0, c=0, arg=0):
    """One Fp operation; mul/inv/div/sqrt/is_qr/pow_u64 on standard form."""
    if op == "add":
        return (a + b) % P, 0
    if op == "sub":
        return (a - b) % P, 0
    if op == "mul":
        return a * b % P, 0
    if op == "neg":
        return (-a) % P, 0
    if op == "inv":
        return _inv0(a), 0
    if op == "div":  # src/fp.cu:571: b == 0 -> 0
        return (a * _inv0(b) % P if b else 0), 0
    if op == "copy":
        return a, 0
    if op == "zero":
        return 0, 0
    if op == "one":
        return 1, 0
    if op == "to_mont":
        return a * R_MONT % P, 0
    if op == "from_mont":
        return a * R_INV % P, 0
    if op == "mont_mul":
        return a * b * R_INV % P, 0
    if op == "cmp":
        return None, (a > b) - (a < b)
    if op == "is_zero":
        return None, int(a == 0)
    if op == "is_one":
        return None, int(a == 1)
    if op == "cmov":
        return (a if arg & 1 else c), 0
    if op == "is_qr":
        return None, int(a == 0 or pow(a, (P - 1) // 2, P) == 1)
    if op == "sqrt":  # src/fp.cu fp_sqrt: a^((p+1)/4), p = 3 mod 4
        if a == 0:
            return 0, 1
        if pow(a, (P - 1) // 2, P) != 1:
            return 0, 0
        r = pow(a, (P + 1) // 4, P)
        if r * r % P == a:
            return r, 1
        alt = (P - r) % P
        return (alt, 1) if alt * alt % P == a else (r, 0)
    if op == "pow_u64":
        return pow(a, arg, P), 0
    raise ValueError(op)


def fp2_elem(op, a=(0, 0), b=(0, 0), c=(0, 0), arg=0):
    """One Fp2 operation; mul/square/inv/div on standard form (src/fp2.cu)."""
    def inv0(x):
        return (0, 0) if x == (0, 0) else f2_inv(x)

    if op == "add":
        return f2_add(a, b), 0
    if op == "sub":
        return f2_sub(a, b), 0
    if op == "mul":
        return f2_mul(a, b), 0
    if op == "square":
        return f2_mul(a, a), 0
    if op == "neg":
        return ((-a[0]) % P, (-a[1]) % P), 0
    if op in ("conjugate", "frobenius"):
        return (a[0], (-a[1]) % P), 0
    if op == "inv":
        return inv0(a), 0
    if op == "div":
        return f2_mul(a, inv0(b)), 0
    if op == "copy":
        return a, 0
    if op == "mul_by_i":
        return ((-a[1]) % P, a[0]), 0
    if op == "cmp":
        d = (a[0] > b[0]) - (a[0] < b[0])
        return None, d if d else (a[1] > b[1]) - (a[1] < b[1])
    if op == "is_zero":
        return None, int(a == (0, 0))
    if op == "is_one":
        return None, int(a == (1, 0))
    if op == "cmov":
        return (a if arg & 1 else c), 0
    if op == "mont_mul":
        m = f2_mul(a, b)
        return (m[0] * R_INV % P, m[1] * R_INV % P), 0
    raise ValueError(op)


def point_elem(op, p, q=None, k=0, group=1):
    """One affine point operation on (x, y, infinity) triples in standard
    form, in the reference's branch order (src/curve.cu:72-268).  Montgomery
    form commutes with these formulas, so the Montgomery-form result is the
    conversion of this one."""
    F = _field(group)
    inf = (F.zero, F.zero, True)

    def inv0(v):
        return F.zero if v == F.zero else F.inv(v)

    def dbl(pt):
        x, y, i = pt
        if i or y == F.zero:
            return inf
        lam = F.mul(inv0(F.add(y, y)), F.add(F.add(F.mul(x, x), F.mul(x, x)), F.mul(x, x)))
        x3 = F.sub(F.mul(lam, lam), F.add(x, x))
        return (x3, F.sub(F.mul(lam, F.sub(x, x3)), y), False)

    def add(p1, p2):
        if p1[2]:
            return p2
        if p2[2]:
            return p1
        (x1, y1, _), (x2, y2, _) = p1, p2
        if x1 == x2 and y1 == F.neg(y2):
            return inf
        if x1 == x2 and y1 == y2:
            return dbl(p1)
        lam = F.mul(inv0(F.sub(x2, x1)), F.sub(y2, y1))
        x3 = F.sub(F.sub(F.mul(lam, lam), x1), x2)
        return (x3, F.sub(F.mul(lam, F.sub(x1, x3)), y1), False)

    if op == "add":
        return add(p, q)
    if op == "double":
        return dbl(p)
    if op == "neg":
        return inf if p[2] else (p[0], F.neg(p[1]), False)
    if op in ("scalar_mul", "scalar_mul_u64"):  # MSB-first double-and-add, src/curve.cu:230
        acc = inf
        if p[2]:
            return inf
        for bit in reversed(range(max(k.bit_length(), 1))):
            acc = dbl(acc)
            if (k >> bit) & 1:
                acc = add(acc, p)
        return acc
    if op == "at_infinity":
        return inf
    raise ValueError(op)
