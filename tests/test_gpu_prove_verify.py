"""prove::prove on the device: fresh blinders, then the self-check
(crates/groth16/src/prove.rs:34-92).  A proof that does not verify against its
own key is refused with SelfVerifyError, as the reference does for a key whose
query sections were tampered with."""
import ctypes

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def key():
    sc = S.SynthCircuit(seed=55, n_constraints=1500, n_inputs=40, n_public=7)
    return sc, sc.zkey(321)


def test_prove_draws_blinders_and_verifies(backend, key):
    sc, zk = key
    ok = O.Zkey(zk)
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    w = sc.witness(1)
    pub = w[32:32 * (1 + ok.n_public)]
    proofs = [circ.prove(w) for _ in range(3)]
    assert len({p.to_bytes() for p in proofs}) == 3          # fresh r, s every call
    for p in proofs:
        assert ok.verify(pub, p.to_bytes())
        circ.verify(pub, p)
    assert circ.stage_timings()["verify_us"] > 0
    with pytest.raises(S.VerifyError):
        circ.verify(sc.witness(2)[32:32 * (1 + ok.n_public)], proofs[0])
    circ.close()


def test_tampered_key_is_refused_by_the_self_check(backend, key):
    sc, zk = key
    pk = S.ProvingKey.from_bytes(zk)
    # shift the L point of a private wire whose value is not zero: the
    # proof's C moves and the proof no longer verifies
    w = sc.witness(1)
    first = pk.n_public + 1
    k = next(i for i in range(pk.n_vars - first) if any(w[32 * (first + i):32 * (first + i + 1)]))
    l0 = pk._view.l_query
    g = S.synth_points(1, 9, 1)
    ctypes.memmove(ctypes.addressof(l0.contents) + 64 * k, g, 64)
    circ = backend.prepare(pk)
    with pytest.raises(S.SelfVerifyError):
        circ.prove(w)
    circ.close()
