"""Batched proving in one launch per stage (g16_prove_batch): every proof of a
submission of mixed circuit sizes, repeated circuits and different tunings
equals the same job proved alone and the oracle's proof, on the first
submission (enqueued stage by stage), on the second (captured as a CUDA graph)
and on the third (the graph replayed); a retuned circuit rebuilds the plan; the
host-lane path (G16_BATCH_ENGINE=0) gives the same proofs."""
import os
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


@pytest.fixture(scope="module")
def mix(backend):
    out = []
    for i, (nc, ni, npub) in enumerate(((90, 8, 2), (700, 20, 4), (4500, 64, 8), (21000, 256, 16))):
        sc = S.SynthCircuit(300 + i, nc, ni, npub)
        zk = sc.zkey(77 + i)
        out.append((sc, zk, O.Zkey(zk), backend.prepare(S.ProvingKey.from_bytes(zk))))
    yield out
    for _, _, ok, c in out:
        c.close()
        ok.close()


def jobs_of(mix, order, seed):
    jobs, meta = [], []
    for k, i in enumerate(order):
        sc, zk, ok, circ = mix[i]
        w = sc.witness(seed + k)
        r, s = blinders(seed + k)
        jobs.append((circ, w, r, s))
        meta.append((ok, w, r, s))
    return jobs, meta


def check(batch, jobs, meta):
    for p, (circ, w, r, s), (ok, _, _, _) in zip(batch, jobs, meta):
        assert p == circ.prove_with_blinders(w, r, s)
        assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        assert ok.verify(w[32:32 * (1 + ok.n_public)], p.to_bytes())


def test_batch_engine_equals_singles_and_oracle(backend, mix):
    order = [0, 1, 2, 3, 3, 2, 1, 0, 2, 2, 1]
    jobs, meta = jobs_of(mix, order, 10)
    launches = S.launch_count()
    done = []
    first = backend.prove_batch(jobs, done_ms=done)
    assert len(done) == len(jobs) and all(d > 0 for d in done)
    check(first, jobs, meta)
    # the same shape twice more: captured, then replayed; different witnesses each time
    for rep in (1, 2):
        jobs2, meta2 = jobs_of(mix, order, 100 * rep)
        check(backend.prove_batch(jobs2), jobs2, meta2)
    assert S.launch_count() > launches


def test_reserved_engines_allocate_nothing(backend, mix):
    # a mix larger than the module's other batches: reserving it sizes every engine,
    # so proving it on whichever engine it lands allocates no device memory
    order = [3, 3, 3, 2, 2, 1, 0, 3, 2, 3, 3, 1]
    before = backend.batch_stats()
    backend.batch_reserve([mix[i][3] for i in order])
    assert backend.batch_stats()["engines"] >= 1
    for rep in range(3):
        jobs, meta = jobs_of(mix, order, 500 + 50 * rep)
        allocs = S.device_alloc_count()
        out = backend.prove_batch(jobs)
        assert S.device_alloc_count() == allocs, "a reserved mix allocated device memory"
        check(out, jobs, meta)
    assert backend.batch_stats()["submissions"] - before["submissions"] == 3


def test_batch_reserve_arguments(backend, mix):
    backend.batch_reserve([])   # nothing to size
    with pytest.raises(S.InvalidArgumentError):
        S.check(S.lib().g16_batch_reserve(None, 0, None))
    with pytest.raises(S.InvalidArgumentError):   # a null circuit
        S.check(S.lib().g16_batch_reserve(backend._h, 1, (S.ctypes.c_void_p * 1)(None)))


def test_batch_engine_after_retuning(backend, mix):
    sc, zk, ok, circ = mix[2]
    t = circ.tuning()
    circ.set_tuning(t["msm_window_bits_witness"] - 1, t["msm_window_bits_h"] + 1, 10, 1)
    try:
        jobs, meta = jobs_of(mix, [2, 3, 2], 500)
        check(backend.prove_batch(jobs), jobs, meta)
    finally:
        circ.set_tuning(t["msm_window_bits_witness"], t["msm_window_bits_h"], t["ntt_tile_log"], t["ntt_outer_log_l"])


def test_batch_lanes_give_the_same_proofs(backend, mix):
    jobs, meta = jobs_of(mix, [3, 0, 1], 900)
    engine = backend.prove_batch(jobs)
    os.environ["G16_BATCH_ENGINE"] = "0"
    try:
        lanes = backend.prove_batch(jobs)
    finally:
        del os.environ["G16_BATCH_ENGINE"]
    assert engine == lanes
    check(engine, jobs, meta)


def test_concurrent_submissions_each_equal_singles(backend, mix):
    """Four threads submit batches of random mixes at once, so several engines
    rebuild layouts and run side by side; every proof equals its single proof."""
    import threading
    refs = {}
    for i in range(len(mix)):
        sc, zk, ok, circ = mix[i]
        for k in range(3):
            w = sc.witness(3000 + 10 * i + k)
            r, s = blinders(4000 + 10 * i + k)
            refs[(i, k)] = (w, r, s, circ.prove_with_blinders(w, r, s))
    bad, errors = [], []

    def worker(tid):
        rng = random.Random(77 + tid)
        try:
            for _ in range(12):
                picks = [(rng.randrange(len(mix)), rng.randrange(3)) for _ in range(rng.randrange(1, 9))]
                jobs = [(mix[i][3],) + refs[(i, k)][:3] for i, k in picks]
                out = backend.prove_batch(jobs)
                bad.extend(q for q, p in zip(picks, out) if p != refs[q][3])
        except Exception as e:   # reported below, on the test's thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert not bad, bad
