"""Host-side check of the device field code's limb arithmetic.

`sqr_redc`, `fq2_mul_redc` and `mul_sub_redc` in snarkrs_b200/csrc/field.cuh
are host-callable: compiled here by nvcc for the CPU, sqr_redc must return
a^2 R^-1 mod p in [0, 2p) for both BN254 moduli (the value the CIOS product
gives before its final conditional subtraction), fq2_mul_redc the two
coordinates of (a0 + a1 u)(b0 + b1 u) R^-1 over Fq[u]/(u^2 + 1), each in
[0, 2q), and mul_sub_redc (a b - c d) R^-1 mod q in [0, 2q), on edge values
and random ones.  The GPU parity tests cover the same
code on the device, bit for bit, through the proofs.
"""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
Q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R_ORDER = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
R = 1 << 256

PROBE = r"""
#include <cstdio>
#include "field.cuh"
// lines of: mode (0 sqr mod q, 1 sqr mod r, 2 Fq2 product, 3 a b - c d mod q), then 1 or 4 operands
// of 8 hex limbs
int main() {
    unsigned a[4][8], r0[8], r1[8];
    int mode;
    while (scanf("%d", &mode) == 1) {
        int n = mode >= 2 ? 4 : 1;
        for (int k = 0; k < n; k++)
            for (int i = 0; i < 8; i++)
                if (scanf("%x", &a[k][i]) != 1) return 1;
        if (mode == 0) g16d::sqr_redc<g16d::FqParams>(a[0], r0);
        else if (mode == 1) g16d::sqr_redc<g16d::FrParams>(a[0], r0);
        else if (mode == 2) g16d::fq2_mul_redc(a[0], a[1], a[2], a[3], r0, r1);
        else g16d::mul_sub_redc<g16d::FqParams>(a[0], a[1], a[2], a[3], r0);
        for (int i = 0; i < 8; i++) printf("%08x ", r0[i]);
        if (mode == 2)
            for (int i = 0; i < 8; i++) printf("%08x ", r1[i]);
        printf("\n");
    }
    return 0;
}
"""


def _limbs(x):
    return " ".join("%x" % ((x >> (32 * i)) & 0xFFFFFFFF) for i in range(8))


def _value(words):
    return sum(int(w, 16) << (32 * i) for i, w in enumerate(words))


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    d = tmp_path_factory.mktemp("field_probe")
    src, exe = d / "probe.cu", d / "probe"
    src.write_text(PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-o", str(exe),
                    str(src)], check=True, capture_output=True)

    def run(lines):
        out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
        return [l.split() for l in out.stdout.split("\n") if l.strip()]
    return run


def test_sqr_redc_matches_big_integers(probe):
    rng = random.Random(20261203)
    cases = []
    for mod, mode in ((Q, 0), (R_ORDER, 1)):
        for a in [0, 1, 2, mod - 1, mod - 2, (mod - 1) // 2] + [rng.randrange(mod) for _ in range(500)]:
            cases.append((a, mod, mode))
    out = probe(["%d %s" % (mode, _limbs(a)) for a, _, mode in cases])
    assert len(out) == len(cases)
    for (a, mod, _), words in zip(cases, out):
        v = _value(words)
        assert v < 2 * mod
        assert v % mod == a * a * pow(R, -1, mod) % mod


def test_fq2_mul_redc_matches_big_integers(probe):
    rng = random.Random(7)
    edge = [0, 1, Q - 1, Q - 2, (Q - 1) // 2]
    cases = [[rng.randrange(Q) for _ in range(4)] for _ in range(500)]
    cases += [[a, b, b, a] for a in edge for b in edge]
    out = probe(["2 " + " ".join(_limbs(x) for x in c) for c in cases])
    assert len(out) == len(cases)
    r_inv = pow(R, -1, Q)
    for (a0, a1, b0, b1), words in zip(cases, out):
        c0, c1 = _value(words[:8]), _value(words[8:])
        assert c0 < 2 * Q and c1 < 2 * Q
        assert c0 % Q == (a0 * b0 - a1 * b1) * r_inv % Q
        assert c1 % Q == (a0 * b1 + a1 * b0) * r_inv % Q


def test_mul_sub_redc_matches_big_integers(probe):
    rng = random.Random(11)
    edge = [0, 1, Q - 1, Q - 2, (Q - 1) // 2]
    cases = [[rng.randrange(Q) for _ in range(4)] for _ in range(500)]
    cases += [[a, b, Q - 1, Q - 1] for a in edge for b in edge] + [[0, 0, a, b] for a in edge for b in edge]
    out = probe(["3 " + " ".join(_limbs(x) for x in c) for c in cases])
    assert len(out) == len(cases)
    r_inv = pow(R, -1, Q)
    for (a, b, c, d), words in zip(cases, out):
        v = _value(words)
        assert v < 2 * Q
        assert v % Q == (a * b - c * d) * r_inv % Q
