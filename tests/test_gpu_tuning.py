"""Per-instance tuning: MSM window sizes and NTT tilings change only the speed.

Every tuning a circuit accepts (set explicitly or chosen by the autotuner)
gives the proof the oracle gives, bit for bit, and the proof passes the
pairing check."""
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def circuit():
    # domain 2^14: inner pass plus outer passes for every tiling tried below
    sc = S.SynthCircuit(seed=77, n_constraints=9000, n_inputs=64, n_public=8)
    zk = sc.zkey(4343)
    return sc, zk, O.Zkey(zk)


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


TUNINGS = [(8, 8, 10, 1), (9, 12, 12, 3), (13, 10, 11, 2), (11, 11, 10, 3), (10, 9, 12, 1), (12, 13, 4, 1)]


def test_every_tuning_gives_the_oracle_proof(backend, circuit):
    sc, zk, ok = circuit
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    model = circ.tuning()
    assert 8 <= model["msm_window_bits_witness"] <= 20 and 8 <= model["msm_window_bits_h"] <= 20
    w = sc.witness(1)
    r, s = blinders(1)
    want = ok.prove(w, O.from_bytes(r), O.from_bytes(s))
    assert circ.prove_with_blinders(w, r, s).to_bytes() == want
    for cw, ch, tl, ll in TUNINGS:
        circ.set_tuning(cw, ch, tl, ll)
        got = circ.tuning()
        assert (got["msm_window_bits_witness"], got["msm_window_bits_h"], got["ntt_tile_log"],
                got["ntt_outer_log_l"]) == (cw, ch, tl, ll)
        for _ in range(2):          # the second proof replays a captured graph
            assert circ.prove_with_blinders(w, r, s).to_bytes() == want
    circ.close()


def test_autotune_keeps_results_and_reports(backend, circuit):
    sc, zk, ok = circuit
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    circ.prove_with_blinders(sc.witness(2), *blinders(2))      # a graph exists before tuning
    t = circ.autotune(sc.witness(3))
    assert t["model_ms"] > 0 and 0 < t["tuned_ms"] <= t["model_ms"]
    assert circ.tuning()["msm_window_bits_witness"] == t["msm_window_bits_witness"]
    for j in (4, 5, 6):
        w = sc.witness(j)
        r, s = blinders(j)
        p = circ.prove_with_blinders(w, r, s).to_bytes()
        assert p == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        assert ok.verify(w[32:32 * (1 + ok.n_public)], p)
    circ.close()


def test_concurrent_autotune_keeps_results(backend, circuit):
    """The batched objective: four proofs in flight on four workspaces."""
    sc, zk, ok = circuit
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    t = circ.autotune(sc.witness(7), concurrency=4)
    assert t["model_ms"] > 0 and 0 < t["tuned_ms"] <= t["model_ms"]
    jobs = []
    for j in (8, 9, 10, 11):
        r, s = blinders(j)
        jobs.append((circ, sc.witness(j), r, s))
    for (c, w, r, s), p in zip(jobs, backend.prove_batch(jobs)):
        assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
    circ.close()


def test_tuning_refusals(backend, circuit):
    sc, zk, _ = circuit
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    for bad in ((7, 10, 11, 2), (10, 21, 11, 2), (10, 10, 13, 2), (10, 10, 11, 11), (10, 10, 1, 0)):
        with pytest.raises(S.InvalidArgumentError):
            circ.set_tuning(*bad)
    with pytest.raises(S.WitnessLengthError):
        circ.autotune(sc.witness(1)[:-32])
    for bad in (0, 9):
        with pytest.raises(S.InvalidArgumentError):
            circ.autotune(sc.witness(1), concurrency=bad)
    circ.close()


def test_warmed_workspaces_allocate_nothing(backend, circuit):
    # g16_circuit_warm readies workspaces with throwaway proofs; real proofs after it
    # allocate no device memory and still equal the oracle's
    sc, zk, ok = circuit
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    try:
        circ.warm(3)
        circ.warm(100)   # more than the pool holds: as many as it can, no error
        held = circ.device_bytes()
        allocs = S.device_alloc_count()
        for i in range(3):
            w = sc.witness(900 + i)
            r, s = blinders(900 + i)
            p = circ.prove_with_blinders(w, r, s)
            assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        assert S.device_alloc_count() == allocs, "a proof on a warmed circuit allocated device memory"
        assert circ.device_bytes() == held
    finally:
        circ.close()
