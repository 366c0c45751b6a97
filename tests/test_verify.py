"""The library's own Groth16 verifier and pairing (host code, no GPU needed).

verify::verify (crates/groth16/src/verify.rs:49-175) is what prove::prove runs
on every proof before returning it.  Here it is checked against the oracle's
independent pairing on the same inputs: the gnark-produced toy proof, proofs
of synthetic circuits made by the oracle prover, tampered proofs, bilinearity,
and the refusals the reference makes (element checks, key checks, counts)."""
import os
import random
import sys

import pytest

import oracle as O
import pyref as P
import snarkrs_b200 as S

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_oracle import _gnark_toy  # noqa: E402


def scalar(k):
    return k.to_bytes(32, "little")


def test_pairing_bilinearity():
    g1 = S.synth_points(1, 5, 1)
    g2 = S.synth_points(2, 6, 1)
    rng = random.Random(1)
    for _ in range(3):
        a, b = rng.randrange(1, O.R_MOD), rng.randrange(1, O.R_MOD)
        aP = O.msm_g1(g1, scalar(a))
        bQ = O.msm_g2(g2, scalar(b))
        neg_abP = O.msm_g1(g1, scalar((-a * b) % O.R_MOD))
        assert S.pairing_check([aP, neg_abP], [bQ, g2])
        wrong = O.msm_g1(g1, scalar((-a * b + 1) % O.R_MOD))
        assert not S.pairing_check([aP, wrong], [bQ, g2])
    # a pair with the point at infinity contributes 1
    assert S.pairing_check([bytes(64)], [g2])
    assert S.pairing_check([], [])
    with pytest.raises(S.InvalidArgumentError):
        S.pairing_check([b"\x01" + bytes(63)], [g2])


def test_gnark_toy_proof():
    vk, (a, b, c), pub = _gnark_toy()
    key = (P.pack_g1(vk["alpha_g1"]), P.pack_g2(vk["beta_g2"]), P.pack_g2(vk["gamma_g2"]),
           P.pack_g2(vk["delta_g2"]), [P.pack_g1(k) for k in vk["k"]])
    proof = P.pack_g1(a) + P.pack_g2(b) + P.pack_g1(c)
    pubm = b"".join(P.fr_to_mont_bytes(x) for x in pub)
    S.verify(key, pubm, proof)
    with pytest.raises(S.VerifyError):
        S.verify(key, b"".join(P.fr_to_mont_bytes((x + 1) % P.R) for x in pub), proof)
    with pytest.raises(S.VerifyError):
        S.verify(key, pubm, P.pack_g1(c) + P.pack_g2(b) + P.pack_g1(a))
    with pytest.raises(S.InvalidArgumentError):
        S.verify(key, pubm + pubm[:32], proof)


@pytest.fixture(scope="module")
def synth():
    sc = S.SynthCircuit(seed=31, n_constraints=400, n_inputs=24, n_public=6)
    zk = sc.zkey(99)
    ok = O.Zkey(zk)
    pk = S.ProvingKey.from_bytes(zk)
    return sc, ok, pk


def test_oracle_proofs_verify_and_tampering_fails(synth):
    sc, ok, pk = synth
    vk = pk.verifying_key()
    rng = random.Random(7)
    for j in range(3):
        w = sc.witness(j)
        r, s = rng.randrange(1, O.R_MOD), rng.randrange(1, O.R_MOD)
        proof = ok.prove(w, O.to_mont(r), O.to_mont(s))
        pub = w[32:32 * (1 + ok.n_public)]
        S.verify(vk, pub, proof)
        assert ok.verify(pub, proof)
        # a different witness's public inputs
        other = sc.witness(j + 10)[32:32 * (1 + ok.n_public)]
        if other != pub:
            with pytest.raises(S.VerifyError):
                S.verify(vk, other, proof)
        # A and C swapped, C replaced by -C
        with pytest.raises(S.VerifyError):
            S.verify(vk, pub, proof[192:] + proof[64:192] + proof[:64])
        neg_c = O.msm_g1(proof[192:], scalar(O.R_MOD - 1))
        with pytest.raises(S.VerifyError):
            S.verify(vk, pub, proof[:192] + neg_c)


def test_element_and_key_refusals(synth):
    sc, ok, pk = synth
    vk = pk.verifying_key()
    w = sc.witness(1)
    proof = ok.prove(w, O.to_mont(5), O.to_mont(7))
    pub = w[32:32 * (1 + ok.n_public)]
    # A at infinity; C off the curve; B off the curve
    for bad in (bytes(64) + proof[64:], proof[:192] + b"\x05" + bytes(63), proof[:64] + b"\x05" + bytes(127) + proof[192:]):
        with pytest.raises(S.VerifyError):
            S.verify(vk, pub, bad)
    # a coordinate not below q
    with pytest.raises(S.VerifyError):
        S.verify(vk, pub, b"\xff" * 64 + proof[64:])
    # gamma == delta: no phase-2 contribution (VerifyingKey::check_structure)
    alpha, beta, gamma, delta, ic = vk
    with pytest.raises(S.FormatError):
        S.verify((alpha, beta, delta, delta, ic), pub, proof)
    with pytest.raises(S.FormatError):
        S.verify((bytes(64), beta, gamma, delta, ic), pub, proof)
    with pytest.raises(S.FormatError):
        S.verify((alpha, beta, gamma, delta, []), b"", proof)
    with pytest.raises(S.InvalidArgumentError):
        S.verify(vk, pub[:-32], proof)


def test_b_outside_the_prime_order_subgroup_is_refused(synth):
    # a point on the twist E'(Fq2) whose order is not r (the twist's cofactor is large):
    # on the curve, so only the subgroup check (verify.rs:57-66) can refuse it, and the
    # refusal names B rather than the pairing
    sc, ok, pk = synth
    vk = pk.verifying_key()
    w = sc.witness(1)
    proof = ok.prove(w, O.to_mont(5), O.to_mont(7))
    pub = w[32:32 * (1 + ok.n_public)]
    k = 1
    while True:
        x = (k, 1)
        y = P.f2_sqrt(P.f2_add(P.f2_mul(P.f2_mul(x, x), x), P.B2))
        if y is not None:
            break
        k += 1
    pt = (x, y)

    def times(p, n):   # n * p without reducing n mod r (P.pt_mul reduces)
        acc = None
        while n:
            if n & 1:
                acc = P.pt_add(acc, p)
            p = P.pt_add(p, p)
            n >>= 1
        return acc
    assert P.on_curve(pt) and times(pt, P.R) is not None
    with pytest.raises(S.VerifyError, match="B is not a valid G2 point"):
        S.verify(vk, pub, proof[:64] + P.pack_g2(pt) + proof[192:])
    # an in-subgroup B that is simply wrong fails the pairing instead
    with pytest.raises(S.VerifyError, match="pairing check failed"):
        S.verify(vk, pub, proof[:64] + P.pack_g2(P.pt_mul(P.G2, 3)) + proof[192:])
