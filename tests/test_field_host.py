"""Host-side check of the device field code's limb arithmetic.

`sqr_redc` in snarkrs_b200/csrc/field.cuh is host-callable: compiled here by
nvcc for the CPU, it must return a^2 R^-1 mod p in [0, 2p) for both BN254
moduli (the value the CIOS product gives before its final conditional
subtraction), on edge values and random ones.  The GPU parity tests cover the
same code on the device, bit for bit, through the proofs.
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
int main() {
    unsigned a[8], r[8];
    int which;
    while (true) {
        for (int i = 0; i < 8; i++)
            if (scanf("%x", &a[i]) != 1) return 0;
        if (scanf("%d", &which) != 1) return 0;
        if (which == 0) g16d::sqr_redc<g16d::FqParams>(a, r);
        else g16d::sqr_redc<g16d::FrParams>(a, r);
        for (int i = 0; i < 8; i++) printf("%08x ", r[i]);
        printf("\n");
    }
}
"""


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_sqr_redc_matches_big_integers(tmp_path):
    src = tmp_path / "sqr_probe.cu"
    exe = tmp_path / "sqr_probe"
    src.write_text(PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-o", str(exe),
                    str(src)], check=True, capture_output=True)
    rng = random.Random(20261203)
    cases = []
    for mod, which in ((Q, 0), (R_ORDER, 1)):
        for a in [0, 1, 2, mod - 1, mod - 2, (mod - 1) // 2, (1 << 254) - 1 if (1 << 254) - 1 < mod else 3] + \
                [rng.randrange(mod) for _ in range(500)]:
            cases.append((a, mod, which))
    text = "\n".join(" ".join("%x" % ((a >> (32 * i)) & 0xFFFFFFFF) for i in range(8)) + " %d" % w
                     for a, _, w in cases) + "\n"
    out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
    for (a, mod, _), line in zip(cases, out):
        v = sum(int(x, 16) << (32 * i) for i, x in enumerate(line.split()))
        assert v < 2 * mod
        assert v % mod == a * a * pow(R, -1, mod) % mod
