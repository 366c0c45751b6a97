"""Pin the CPU oracle before trusting it: reference golden constants, the gnark
toy proof, an independent pure-Python big-integer restatement, and the
algebraic identities every Groth16 proof must satisfy.  CPU only."""
import json
import os
import random

import pytest

import oracle as O
import pyref as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_reference_constants():
    """crates/gpu-layout/src/lib.rs:80-113, 526-540; crates/groth16/src/prove.rs:549-563."""
    g = golden("reference_constants.json")
    p, n0, one, _ = O.field_consts(0)
    assert p == int(g["fr_modulus"]) == O.R_MOD
    assert (n0 & 0xFFFFFFFF) == g["fr_n0_u32"]
    assert one == int(g["fr_r_mod_r"])
    q, n0q, _, _ = O.field_consts(1)
    assert q == int(g["fq_modulus"]) == O.Q_MOD
    assert (n0q & 0xFFFFFFFF) == g["fq_n0_u32"]
    assert O.from_mont(O.domain_root(28)) == int(g["domain_root_2_28"])
    assert O.from_mont(O.domain_root(4)) == int(g["domain_root_2_4"])


def test_coset_shift_identities():
    """shift^2 = omega_n and shift^n = -1 (crates/groth16/src/cpu.rs:915-927)."""
    R = O.R_MOD
    for log_n in (1, 3, 10, 16, 27):
        w = O.from_mont(O.domain_root(log_n))
        shift = O.from_mont(O.domain_root(log_n + 1))
        assert shift * shift % R == w
        assert pow(shift, 1 << log_n, R) == R - 1
        assert pow(w, 1 << log_n, R) == 1
        if log_n:
            assert pow(w, 1 << (log_n - 1), R) != 1


def test_field_matches_python():
    rng = random.Random(3)
    for which, M in ((0, O.R_MOD), (1, O.Q_MOD)):
        edge = [0, 1, 2, M - 1, M - 2, (M - 1) // 2, 1 << 128, (1 << 253) % M]
        vals = edge + [rng.randrange(M) for _ in range(300)]
        for a in vals:
            b = rng.choice(vals)
            am, bm = O.to_mont(a, M), O.to_mont(b, M)
            assert O.from_mont(O.fp_op("mul", which, am, bm), M) == a * b % M
            assert O.from_mont(O.fp_op("add", which, am, bm), M) == (a + b) % M
            assert O.from_mont(O.fp_op("sub", which, am, bm), M) == (a - b) % M
            if a:
                assert O.from_mont(O.fp_op("inv", which, am), M) == pow(a, -1, M)


def test_fq2_matches_python():
    rng = random.Random(4)
    Q = O.Q_MOD
    for _ in range(100):
        a = (rng.randrange(Q), rng.randrange(Q))
        b = (rng.randrange(Q), rng.randrange(Q))
        got = O.fq2_mul((O.to_mont(a[0], Q), O.to_mont(a[1], Q)), (O.to_mont(b[0], Q), O.to_mont(b[1], Q)))
        assert (O.from_mont(got[0], Q), O.from_mont(got[1], Q)) == P.f2_mul(a, b)


def test_hard_exponent():
    assert O.hard_exponent() == (O.Q_MOD ** 4 - O.Q_MOD ** 2 + 1) // O.R_MOD


def _dft(vals, w, R):
    n = len(vals)
    return [sum(v * pow(w, i * j, R) for j, v in enumerate(vals)) % R for i in range(n)]


@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8])
def test_ntt_matches_naive_dft(log_n):
    """CpuNtt::ntt equals the DFT (crates/ntt/src/lib.rs:1298 naive DFT test)."""
    R = O.R_MOD
    n = 1 << log_n
    rng = random.Random(log_n)
    vals = [rng.randrange(R) for _ in range(n)]
    data = b"".join(O.to_bytes(O.to_mont(v)) for v in vals)
    w = O.from_mont(O.domain_root(log_n))
    out = O.ntt(log_n, O.NTT_FORWARD, data)
    got = [O.from_mont(O.from_bytes(out[32 * i:32 * i + 32])) for i in range(n)]
    assert got == _dft(vals, w, R)
    back = O.ntt(log_n, O.NTT_INVERSE, out)
    assert back == data
    # intt_coset_ntt: evaluations on the odd coset of the interpolant
    shift = O.from_mont(O.domain_root(log_n + 1))
    coeffs = [v * pow(n, -1, R) % R for v in _dft(vals, pow(w, -1, R), R)]
    ev = [sum(c * pow(shift * pow(w, i, R), j, R) for j, c in enumerate(coeffs)) % R for i in range(n)]
    out = O.ntt(log_n, O.NTT_INTT_COSET_NTT, data)
    assert [O.from_mont(O.from_bytes(out[32 * i:32 * i + 32])) for i in range(n)] == ev


def test_g1_g2_scalar_mul_matches_python():
    rng = random.Random(5)
    G1, G2 = O.g1_generator(), O.g2_generator()
    assert P.unpack_g1(G1) == P.G1 and P.unpack_g2(G2) == P.G2
    for k in [0, 1, 2, O.R_MOD - 1, rng.randrange(O.R_MOD)]:
        assert P.unpack_g1(O.g1_mul(G1, k)) == P.pt_mul(P.G1, k)
    for k in [1, 3, rng.randrange(O.R_MOD)]:
        assert P.unpack_g2(O.g2_mul(G2, k)) == P.pt_mul(P.G2, k)
    assert O.g1_mul(G1, O.R_MOD) == bytes(64)   # r G = infinity


def test_msm_matches_naive_with_edge_cases():
    """Pippenger vs a naive sum: zeros, ones, infinity bases, repeated and opposite bases."""
    rng = random.Random(6)
    R = O.R_MOD
    pts = [P.pt_mul(P.G1, rng.randrange(1, R)) for _ in range(12)]
    pts[3] = None                      # infinity base
    pts[5] = pts[4]                    # repeated base (bucket doubling)
    pts[7] = P.pt_neg(pts[6])          # opposite bases (cancellation)
    ks = [rng.randrange(R) for _ in pts]
    ks[0], ks[1], ks[2] = 0, 1, R - 1
    ks[5] = ks[4]
    ks[7] = ks[6]
    bases = b"".join(P.pack_g1(p) for p in pts)
    scal = b"".join(k.to_bytes(32, "little") for k in ks)
    assert P.unpack_g1(O.msm_g1(bases, scal)) == P.msm_naive(pts, ks)
    pts2 = [P.pt_mul(P.G2, rng.randrange(1, R)) for _ in range(5)]
    ks2 = [rng.randrange(R) for _ in pts2]
    got = O.msm_g2(b"".join(P.pack_g2(p) for p in pts2), b"".join(k.to_bytes(32, "little") for k in ks2))
    assert P.unpack_g2(got) == P.msm_naive(pts2, ks2)


def test_msm_larger_against_split_sums():
    """A few thousand points: the MSM is linear, so MSM(a) + MSM(b) = MSM(a + b)."""
    rng = random.Random(8)
    R = O.R_MOD
    n = 3000
    base_k = [rng.randrange(1, R) for _ in range(n)]
    bases = b"".join(O.g1_mul(O.g1_generator(), k) for k in base_k[:64]) * (n // 64) + \
        b"".join(O.g1_mul(O.g1_generator(), k) for k in base_k[:n % 64])
    a = [rng.randrange(R) for _ in range(n)]
    b = [rng.randrange(R) for _ in range(n)]
    enc = lambda v: b"".join(x.to_bytes(32, "little") for x in v)
    lhs = O.g1_add(O.msm_g1(bases, enc(a)), O.msm_g1(bases, enc(b)))
    rhs = O.msm_g1(bases, enc([(x + y) % R for x, y in zip(a, b)]))
    assert lhs == rhs
    # and against the discrete-log form: sum k_i a_i G
    logs = (base_k[:64] * (n // 64 + 1))[:n]
    want = O.g1_mul(O.g1_generator(), sum(x * y for x, y in zip(logs, a)) % R)
    assert O.msm_g1(bases, enc(a)) == want


def test_pairing_bilinear():
    rng = random.Random(9)
    R = O.R_MOD
    a, b = rng.randrange(1, R), rng.randrange(1, R)
    P1, Q2 = O.g1_mul(O.g1_generator(), a), O.g2_mul(O.g2_generator(), b)
    neg = O.g1_mul(O.g1_generator(), (-a * b) % R)
    assert O.pairing_check([P1, neg], [Q2, O.g2_generator()])
    assert not O.pairing_check([P1, O.g1_mul(O.g1_generator(), (-a * b + 1) % R)], [Q2, O.g2_generator()])


def _gnark_toy():
    toy = golden("gnark_toy.json")
    vk = P.gnark_vk(bytes.fromhex(toy["vk.bin"]))
    a, b, c = P.gnark_proof(bytes.fromhex(toy["proof.bin"]))
    pub = P.gnark_public(bytes.fromhex(toy["public.bin"]))
    return vk, (a, b, c), pub


def test_gnark_toy_proof_verifies():
    """The committed gnark v0.14 proof (test-support/gnark/toy) must pass an independent pairing."""
    vk, (a, b, c), pub = _gnark_toy()
    proof = P.pack_g1(a) + P.pack_g2(b) + P.pack_g1(c)
    pubm = b"".join(P.fr_to_mont_bytes(x) for x in pub)
    args = (P.pack_g1(vk["alpha_g1"]), P.pack_g2(vk["beta_g2"]), P.pack_g2(vk["gamma_g2"]),
            P.pack_g2(vk["delta_g2"]), [P.pack_g1(k) for k in vk["k"]])
    assert O.verify_vk(*args, pubm, proof)
    bad = b"".join(P.fr_to_mont_bytes((x + 1) % P.R) for x in pub)
    assert not O.verify_vk(*args, bad, proof)
    swapped = P.pack_g1(c) + P.pack_g2(b) + P.pack_g1(a)
    assert not O.verify_vk(*args, pubm, swapped)


def test_rows_path_restatement_matches_compute_h():
    """h_and_msms_from_rows (crates/groth16/src/cpu.rs:384-425): the witness's own rows,
    whole or cut after the last nonzero row, give the H of compute_h."""
    import snarkrs_b200 as S
    sc = S.SynthCircuit(seed=13, n_constraints=500, n_inputs=20, n_public=4)
    ok = O.Zkey(sc.zkey(77))
    w = sc.witness(2)
    a, b = ok.gather(w)
    h = ok.compute_h(w)
    assert ok.compute_h_from_rows(a, b) == h
    n = len(a) // 32
    last = max(i for i in range(n) if any(a[32 * i:32 * i + 32]) or any(b[32 * i:32 * i + 32]))
    assert ok.compute_h_from_rows(a[:32 * (last + 1)], b[:32 * (last + 1)]) == h
    # rows that are not the witness's give another H
    bad = bytearray(a)
    bad[0] ^= 1
    assert ok.compute_h_from_rows(bytes(bad), b) != h
