"""The gnark key on the B200 (HBasis::GnarkBitReversed, crates/groth16/src/lib.rs:425-444,
cpu.rs:384-471): the committed gnark toy key and witness rows prove bit-exactly
the oracle's proof, which verifies under gnark's verifying key; the same with a
compact key; the gather-path entry points refuse a key without matrices."""
import gzip
import json
import os
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture(name):
    with gzip.open(os.path.join(HERE, "golden", name)) as f:
        return f.read()


@pytest.fixture(scope="module")
def toy():
    with open(os.path.join(HERE, "golden", "gnark_toy.json")) as f:
        vk = bytes.fromhex(json.load(f)["vk.bin"])
    pk = fixture("gnark_toy_pk.dump.gz")
    w, aw, bw = S.gnark_witness(fixture("gnark_toy_witness.bin.gz"))
    ok = O.Zkey.from_gnark(pk, vk)
    yield pk, vk, w, aw, bw, ok
    ok.close()


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


def test_gnark_rows_prove_equals_oracle(backend, toy):
    pk, vk, w, aw, bw, ok = toy
    c = backend.prepare(S.ProvingKey.from_gnark(pk, vk))
    pub = w[32:32 * (1 + ok.n_public)]
    for seed in (1, 2, 3):
        r, s = blinders(seed)
        p = c.prove_with_blinders_from_rows(w, aw, bw, r, s)
        assert p.to_bytes() == ok.prove_rows(w, aw, bw, O.from_bytes(r), O.from_bytes(s))
        c.verify(pub, p)
        assert ok.verify(pub, p.to_bytes())
    # fewer rows than the domain, zero padded (the rows are one per constraint)
    assert len(aw) // 32 < c.domain_size
    # the gather path needs constraint matrices the key does not have
    r, s = blinders(9)
    for call in (lambda: c.prove_with_blinders(w, r, s), lambda: c.compute_h(w),
                 lambda: backend.prove_batch([(c, w, r, s)])):
        with pytest.raises(S.BackendError, match="rows"):
            call()
    c.close()


def test_gnark_compact_key(backend, toy):
    pk, vk, w, aw, bw, ok = toy
    os.environ["G16_CUDA_WINDOW_TABLES"] = "0"
    try:
        c = backend.prepare(S.ProvingKey.from_gnark(pk, vk))
    finally:
        del os.environ["G16_CUDA_WINDOW_TABLES"]
    assert not c.window_tables()
    r, s = blinders(4)
    p = c.prove_with_blinders_from_rows(w, aw, bw, r, s)
    assert p.to_bytes() == ok.prove_rows(w, aw, bw, O.from_bytes(r), O.from_bytes(s))
    c.close()
