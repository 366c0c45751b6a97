"""A slow, independent pure-Python BN254 reference used to pin the C oracle.

Python integers make the field arithmetic obviously correct; the group law is
the textbook affine one.  Only small cases run through here.  Also holds the
gnark v0.14 point decoders (restating crates/gnark/src/lib.rs:159-306) so the
committed gnark toy fixture can be fed to the oracle's pairing check.
"""
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
MONT = 1 << 256

G1 = (1, 2)
G2 = ((10857046999023057135944570762232829481370756359578518086990519993285655852781,
       11559732032986387107991004021392285783925812861821192530917403151452391805634),
      (8495653923123431417604973247489272438418190587263600148770280649306958101930,
       4082367875863433681332203403145435568316851327593401208105741076214120093531))


# ---------------- Fq2 = Fq[u]/(u^2+1), elements are (c0, c1) ----------------
def f2_add(a, b):
    return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)


def f2_sub(a, b):
    return ((a[0] - b[0]) % Q, (a[1] - b[1]) % Q)


def f2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def f2_neg(a):
    return ((-a[0]) % Q, (-a[1]) % Q)


def f2_inv(a):
    n = pow(a[0] * a[0] + a[1] * a[1], Q - 2, Q)
    return (a[0] * n % Q, (-a[1] * n) % Q)


def f2_pow(a, e):
    acc = (1, 0)
    while e:
        if e & 1:
            acc = f2_mul(acc, a)
        a = f2_mul(a, a)
        e >>= 1
    return acc


def f2_sqrt(a):
    """Square root for q = 3 mod 4 (Adj & Rodriguez-Henriquez, Algorithm 9)."""
    if a == (0, 0):
        return (0, 0)
    a1 = f2_pow(a, (Q - 3) // 4)
    alpha = f2_mul(f2_mul(a1, a), a1)
    a0 = f2_mul((alpha[0], (-alpha[1]) % Q), alpha)
    if a0 == (Q - 1, 0):
        return None
    x0 = f2_mul(a1, a)
    if alpha == (Q - 1, 0):
        x = f2_mul((0, 1), x0)
    else:
        b = f2_pow(f2_add((1, 0), alpha), (Q - 1) // 2)
        x = f2_mul(b, x0)
    return x if f2_mul(x, x) == a else None


XI = (9, 1)
B2 = f2_mul((3, 0), f2_inv(XI))


# ---------------- generic affine group law (None = infinity) ----------------
class Field1:
    add = staticmethod(lambda a, b: (a + b) % Q)
    sub = staticmethod(lambda a, b: (a - b) % Q)
    mul = staticmethod(lambda a, b: a * b % Q)
    inv = staticmethod(lambda a: pow(a, Q - 2, Q))
    neg = staticmethod(lambda a: (-a) % Q)
    zero = 0
    three = 3


class Field2:
    add = staticmethod(f2_add)
    sub = staticmethod(f2_sub)
    mul = staticmethod(f2_mul)
    inv = staticmethod(f2_inv)
    neg = staticmethod(f2_neg)
    zero = (0, 0)
    three = (3, 0)


def _field(p):
    return Field2 if isinstance(p[0], tuple) else Field1


def pt_add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    F = _field(p)
    if p[0] == q[0]:
        if F.add(p[1], q[1]) == F.zero:
            return None
        lam = F.mul(F.mul(F.three, F.mul(p[0], p[0])), F.inv(F.add(p[1], p[1])))
    else:
        lam = F.mul(F.sub(q[1], p[1]), F.inv(F.sub(q[0], p[0])))
    x3 = F.sub(F.sub(F.mul(lam, lam), p[0]), q[0])
    y3 = F.sub(F.mul(lam, F.sub(p[0], x3)), p[1])
    return (x3, y3)


def pt_neg(p):
    return None if p is None else (p[0], _field(p).neg(p[1]))


def pt_mul(p, k):
    k %= R
    acc = None
    while k:
        if k & 1:
            acc = pt_add(acc, p)
        p = pt_add(p, p)
        k >>= 1
    return acc


def msm_naive(points, scalars):
    acc = None
    for p, k in zip(points, scalars):
        acc = pt_add(acc, pt_mul(p, k))
    return acc


def on_curve(p):
    if p is None:
        return True
    F = _field(p)
    b = 3 if F is Field1 else B2
    return F.mul(p[1], p[1]) == F.add(F.mul(F.mul(p[0], p[0]), p[0]), b)


# ---------------- packed byte layout (Montgomery LE, infinity = zeros) ----------------
def fq_to_mont_bytes(x):
    return ((x * MONT) % Q).to_bytes(32, "little")


def fq_from_mont_bytes(b):
    return int.from_bytes(b, "little") * pow(MONT, -1, Q) % Q


def pack_g1(p):
    if p is None:
        return bytes(64)
    return fq_to_mont_bytes(p[0]) + fq_to_mont_bytes(p[1])


def pack_g2(p):
    if p is None:
        return bytes(128)
    return b"".join(fq_to_mont_bytes(c) for c in (p[0][0], p[0][1], p[1][0], p[1][1]))


def unpack_g1(b):
    if b == bytes(64):
        return None
    return (fq_from_mont_bytes(b[:32]), fq_from_mont_bytes(b[32:64]))


def unpack_g2(b):
    if b == bytes(128):
        return None
    c = [fq_from_mont_bytes(b[32 * i:32 * i + 32]) for i in range(4)]
    return ((c[0], c[1]), (c[2], c[3]))


def fr_to_mont_bytes(x):
    return ((x * MONT) % R).to_bytes(32, "little")


# ---------------- gnark v0.14 encoder points ----------------
_FLAG_MASK = 0b11 << 6
_UNCOMPRESSED, _INF, _SMALL, _LARGE = 0, 0b01 << 6, 0b10 << 6, 0b11 << 6


def _fq_largest(y):
    return y > (Q - 1) // 2


def _fq2_largest(y):
    return _fq_largest(y[0]) if y[1] == 0 else _fq_largest(y[1])


def gnark_g1(b, off):
    """Decode one encoder G1 point at ``off``; returns (point, new offset)."""
    flag = b[off] & _FLAG_MASK
    xb = bytes([b[off] & ~_FLAG_MASK & 0xFF]) + b[off + 1:off + 32]
    if flag == _UNCOMPRESSED:
        raw = b[off:off + 64]
        if raw == bytes(64):
            return None, off + 64
        return (int.from_bytes(xb, "big"), int.from_bytes(raw[32:], "big")), off + 64
    if flag == _INF:
        return None, off + 32
    x = int.from_bytes(xb, "big")
    y2 = (x * x * x + 3) % Q
    y = pow(y2, (Q + 1) // 4, Q)
    assert y * y % Q == y2, "not on curve"
    if _fq_largest(y) != (flag == _LARGE):
        y = (-y) % Q
    return (x, y), off + 32


def gnark_g2(b, off):
    flag = b[off] & _FLAG_MASK
    x1b = bytes([b[off] & ~_FLAG_MASK & 0xFF]) + b[off + 1:off + 32]
    if flag == _UNCOMPRESSED:
        raw = b[off:off + 128]
        if raw == bytes(128):
            return None, off + 128
        x1 = int.from_bytes(x1b, "big")
        x0, y1, y0 = (int.from_bytes(raw[32 * i:32 * i + 32], "big") for i in (1, 2, 3))
        return ((x0, x1), (y0, y1)), off + 128
    if flag == _INF:
        return None, off + 64
    x = (int.from_bytes(b[off + 32:off + 64], "big"), int.from_bytes(x1b, "big"))
    y2 = f2_add(f2_mul(f2_mul(x, x), x), B2)
    y = f2_sqrt(y2)
    assert y is not None, "not on curve"
    if _fq2_largest(y) != (flag == _LARGE):
        y = f2_neg(y)
    return (x, y), off + 64


def gnark_vk(b):
    off = 0
    alpha, off = gnark_g1(b, off)
    beta1, off = gnark_g1(b, off)
    beta2, off = gnark_g2(b, off)
    gamma2, off = gnark_g2(b, off)
    delta1, off = gnark_g1(b, off)
    delta2, off = gnark_g2(b, off)
    nk = int.from_bytes(b[off:off + 4], "big")
    off += 4
    k = []
    for _ in range(nk):
        p, off = gnark_g1(b, off)
        k.append(p)
    return {"alpha_g1": alpha, "beta_g1": beta1, "beta_g2": beta2, "gamma_g2": gamma2,
            "delta_g1": delta1, "delta_g2": delta2, "k": k}


def gnark_proof(b):
    a, off = gnark_g1(b, 0)
    bb, off = gnark_g2(b, off)
    c, off = gnark_g1(b, off)
    return a, bb, c


def gnark_public(b):
    return [int.from_bytes(b[i:i + 32], "big") for i in range(0, len(b), 32)]
