"""The timed CPU baseline (oracle/port_*.c) and the oracle's own input generator
(oracle/synth.c), checked on the CPU.

The baseline restates the reference CPU prover's fast algorithms (batch-affine
MSM fill, the five MSMs concurrently, the 2^11-blocked intt_coset_ntt), and
its results must equal the plain oracle's bit for bit: field products, the
prover's NTT chain, MSMs (edge cases included) and whole proofs.  The oracle's
generator must give the same circuit, witnesses and .zkey bytes as the
product's, so that the reference arm can run without the product library."""
import random

import pytest

import oracle as O
import pyref as P
import snarkrs_b200 as S


def test_port_field_products_match_the_oracle():
    import ctypes
    rng = random.Random(11)
    L = O.lib()
    for which, mod in ((0, O.R_MOD), (1, O.Q_MOD)):
        vals = [0, 1, mod - 1, mod - 2] + [rng.randrange(mod) for _ in range(1500)]
        for a, b in zip(vals, reversed(vals)):
            out = ctypes.create_string_buffer(32)
            L.oracle_port_fp_mul(which, O.to_bytes(a), O.to_bytes(b), out)
            assert O.from_bytes(out.raw) == O.fp_op("mul", which, a, b)
    for a in [1, 2, O.Q_MOD - 1] + [rng.randrange(1, O.Q_MOD) for _ in range(20)]:
        out = ctypes.create_string_buffer(32)
        L.oracle_port_fq_inv(O.to_bytes(a), out)
        assert O.from_bytes(out.raw) == O.fp_op("inv", 1, a)


@pytest.mark.parametrize("log_n", [1, 2, 5, 10, 11, 12, 13, 14])
def test_port_intt_coset_ntt_matches_the_oracle(log_n):
    rng = random.Random(log_n)
    data = b"".join(O.to_bytes(rng.randrange(O.R_MOD)) for _ in range(1 << log_n))
    assert O.port_intt_coset_ntt(log_n, data) == O.ntt(log_n, O.NTT_INTT_COSET_NTT, data)


@pytest.mark.parametrize("n,dist", [(1, 0), (5, 1), (300, 0), (3000, 1), (20000, 0), (60000, 1)])
def test_port_msm_g1_matches_the_oracle(n, dist):
    b, s = S.synth_points(1, 40 + n, n), S.synth_scalars(41 + n, n, dist)
    assert O.port_msm_g1(b, s) == O.msm_g1(b, s)


@pytest.mark.parametrize("n,dist", [(3, 0), (700, 1), (5000, 0)])
def test_port_msm_g2_matches_the_oracle(n, dist):
    b, s = S.synth_points(2, 50 + n, n), S.synth_scalars(51 + n, n, dist)
    assert O.port_msm_g2(b, s) == O.msm_g2(b, s)


def test_port_msm_edge_cases():
    """Zeros, ones, r-1, infinity bases, P+P and P-P in one bucket, one scalar over many
    bases (every addition a batch conflict: the retry and XYZZ side-bucket paths)."""
    rng = random.Random(3)
    pts = [P.pt_mul(P.G1, rng.randrange(1, O.R_MOD)) for _ in range(60)]
    pts[3] = None
    pts[5] = pts[4]
    pts[7] = P.pt_neg(pts[6])
    ks = [rng.randrange(O.R_MOD) for _ in pts]
    ks[0], ks[1], ks[2] = 0, 1, O.R_MOD - 1
    ks[5], ks[7] = ks[4], ks[6]
    bases = b"".join(P.pack_g1(p) for p in pts)
    scal = b"".join(k.to_bytes(32, "little") for k in ks)
    assert O.port_msm_g1(bases, scal) == O.msm_g1(bases, scal) == P.pack_g1(P.msm_naive(pts, ks))
    assert O.port_msm_g1(bases, bytes(32 * len(pts))) == bytes(64)
    n = 4000
    b = S.synth_points(1, 8, n)
    k = rng.randrange(O.R_MOD).to_bytes(32, "little")
    assert O.port_msm_g1(b, k * n) == O.msm_g1(b, k * n)
    neg = (O.R_MOD - int.from_bytes(k, "little")).to_bytes(32, "little")
    assert O.port_msm_g1(b + b, k * n + neg * n) == bytes(64)


@pytest.mark.parametrize("nc", [150, 3000, 20000])
def test_port_proofs_equal_the_oracles(nc):
    sc = O.Synth(60 + nc, nc, 32, 4)
    zk = sc.zkey(8)
    ok = O.Zkey(zk)
    port = O.PortProver(ok)
    rng = random.Random(nc)
    for ws in (1, 2):
        w = sc.witness(ws)
        r, s = rng.randrange(1, O.R_MOD), rng.randrange(1, O.R_MOD)
        got = port.prove(w, O.to_bytes(O.to_mont(r)), O.to_bytes(O.to_mont(s)))
        assert got == ok.prove(w, O.to_mont(r), O.to_mont(s))
        assert ok.verify(w[32:32 * (1 + ok.n_public)], got)
    port.close()


@pytest.mark.parametrize("seed,nc,ni,npub", [(1, 300, 20, 4), (7, 5000, 64, 8), (21, 30000, 256, 16)])
def test_oracle_generator_gives_the_products_bytes(seed, nc, ni, npub):
    mine = O.Synth(seed, nc, ni, npub)
    theirs = S.SynthCircuit(seed, nc, ni, npub)
    assert (mine.n_vars, mine.domain_size) == (theirs.n_vars, theirs.domain_size)
    for ws in (0, 99):
        assert mine.witness(ws) == theirs.witness(ws)
    assert mine.zkey(5) == theirs.zkey(5)
