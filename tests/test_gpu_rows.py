"""PreparedCircuit::h_and_msms_from_rows on the device (crates/groth16/src/lib.rs:425-444,
crates/groth16/src/cpu.rs:384-471): stage 0 handed over as A.w and B.w rows."""
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(backend):
    sc = S.SynthCircuit(seed=99, n_constraints=2500, n_inputs=48, n_public=6)
    zk = sc.zkey(1234)
    ok = O.Zkey(zk)
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    yield sc, ok, circ
    circ.close()


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


def last_row(a, b):
    n = len(a) // 32
    return max(i for i in range(n) if any(a[32 * i:32 * i + 32]) or any(b[32 * i:32 * i + 32])) + 1


def test_rows_match_the_gather_path_and_the_oracle(setup):
    sc, ok, circ = setup
    w = sc.witness(1)
    a, b = ok.gather(w)
    want = circ.h_and_msms(w).as_dict()
    assert circ.h_and_msms_from_rows(w, a, b).as_dict() == want
    k = last_row(a, b)
    assert circ.h_and_msms_from_rows(w, a[:32 * k], b[:32 * k]).as_dict() == want
    assert want == ok.msms(w, ok.compute_h_from_rows(a[:32 * k], b[:32 * k]))


def test_prove_from_rows_equals_prove_and_verifies(setup):
    sc, ok, circ = setup
    w = sc.witness(2)
    a, b = ok.gather(w)
    r, s = blinders(2)
    p = circ.prove_with_blinders_from_rows(w, a, b, r, s)
    assert p == circ.prove_with_blinders(w, r, s)
    assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
    circ.verify(w[32:32 * (1 + ok.n_public)], p)
    # rows that are not this witness's: the proof does not verify (prove.rs:93-101)
    bad = bytearray(a)
    bad[32 * 7] ^= 1
    q = circ.prove_with_blinders_from_rows(w, bytes(bad), b, r, s)
    with pytest.raises(S.VerifyError):
        circ.verify(w[32:32 * (1 + ok.n_public)], q)


def test_rows_refusals(setup):
    sc, ok, circ = setup
    w = sc.witness(3)
    a, b = ok.gather(w)
    with pytest.raises(S.BackendError):
        circ.h_and_msms_from_rows(w, a + a[:32], b + b[:32])      # more rows than the domain
    with pytest.raises(S.BackendError):
        circ.h_and_msms_from_rows(w, a, b[:-32])
    with pytest.raises(S.WitnessLengthError):
        circ.h_and_msms_from_rows(w[:-32], a, b)
