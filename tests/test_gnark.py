"""gnark v0.14 keys on the host (crates/gnark): the product's reader and the
oracle's independent one agree on every query of the committed gnark toy key
(tests/golden/gnark_toy_pk.dump.gz, its verifying key in gnark_toy.json), the
witness dump's W, A.w and B.w agree, malformed files are refused, and the
oracle's proof from the key and the witness rows -- gnark's bit-reversed H
basis -- verifies under gnark's own verifying key with both verifiers."""
import gzip
import json
import os
import random

import pytest

import oracle as O
import pyref as P
import snarkrs_b200 as S

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture(name):
    with gzip.open(os.path.join(HERE, "golden", name)) as f:
        return f.read()


@pytest.fixture(scope="module")
def toy():
    with open(os.path.join(HERE, "golden", "gnark_toy.json")) as f:
        j = json.load(f)
    return fixture("gnark_toy_pk.dump.gz"), bytes.fromhex(j["vk.bin"]), fixture("gnark_toy_witness.bin.gz"), j


def test_readers_agree(toy):
    pk, vk, wit, _ = toy
    k = S.ProvingKey.from_gnark(pk, vk)
    ok = O.Zkey.from_gnark(pk, vk)
    assert k.gnark and ok.gnark
    assert (k.n_vars, k.n_public, k.domain_size) == (ok.n_vars, ok.n_public, ok.domain_size) == (3072, 4, 4096)
    for mine, theirs in (("a_query", "a"), ("b_g1_query", "b1"), ("b_g2_query", "b2"), ("l_query", "l"),
                         ("h_query", "h")):
        assert k.query_bytes(mine) == ok.query(theirs), mine
    alpha, beta, gamma, delta, ic = k.verifying_key()
    assert alpha + beta + gamma + delta + b"".join(ic) == ok.vk_bytes()
    assert len(k.query_bytes("h_query")) == 64 * (k.domain_size - 1)
    w, aw, bw = S.gnark_witness(wit)
    assert (w, aw, bw) == O.gnark_witness(wit)
    assert len(w) // 32 == k.n_vars and len(aw) == len(bw) == 32 * 2071
    ok.close()


def test_header_points_match_an_independent_decoder(toy):
    pk, vk, _, j = toy
    k = S.ProvingKey.from_gnark(pk, vk)
    ref = P.gnark_vk(vk)
    alpha, beta, gamma, delta, ic = k.verifying_key()

    def g1(b):
        return (O.from_mont(O.from_bytes(b[:32]), P.Q), O.from_mont(O.from_bytes(b[32:]), P.Q))

    assert g1(alpha) == ref["alpha_g1"]
    assert [g1(p) for p in ic] == ref["k"]


def test_malformed_files_are_refused(toy):
    pk, vk, wit, _ = toy
    for bad in (pk[:-1], b"\0" * 8 + pk[8:], pk[:100]):
        with pytest.raises(S.FormatError):
            S.ProvingKey.from_gnark(bad, vk)
    # a verifying key whose alpha differs (flip a bit of x: off the curve or another point)
    vb = bytearray(vk)
    vb[31] ^= 1
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_gnark(pk, bytes(vb))
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_gnark(pk, vk + b"\0")
    # a commitment key count
    off = 8 + 8 + 5 * 32 + 1 + 3 * 64 + 2 * 128 + 24 + 2 * 3072
    pb = bytearray(pk)
    pb[off + 3] = 1
    with pytest.raises(S.FormatError, match="commitment"):
        S.ProvingKey.from_gnark(bytes(pb), vk)
    with pytest.raises(S.FormatError):
        S.gnark_witness(wit[:-5])


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


def test_oracle_proves_with_the_gnark_key(toy):
    pk, vk, wit, j = toy
    ok = O.Zkey.from_gnark(pk, vk)
    w, aw, bw = O.gnark_witness(wit)
    r, s = blinders(11)
    proof = ok.prove_rows(w, aw, bw, O.from_bytes(r), O.from_bytes(s))
    pub = w[32:32 * (1 + ok.n_public)]
    assert ok.verify(pub, proof)
    # the product's host verifier, against the verifying key gnark wrote
    k = S.ProvingKey.from_gnark(pk, vk)
    S.verify(k.verifying_key(), pub, S.Proof(proof[:64], proof[64:192], proof[192:]))
    # the public inputs are the ones gnark's own proof verifies with
    assert [int.from_bytes(bytes.fromhex(j["public.bin"])[i:i + 32], "big") for i in range(0, 128, 32)] == \
        [O.from_mont(O.from_bytes(pub[i:i + 32])) for i in range(0, len(pub), 32)]
    # a wrong row gives a proof that does not verify
    bad = bytearray(aw)
    bad[0] ^= 1
    assert not ok.verify(pub, ok.prove_rows(w, bytes(bad), bw, O.from_bytes(r), O.from_bytes(s)))
    ok.close()
