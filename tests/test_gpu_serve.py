"""Served proving (continuous batching, LRU key residency): every proof equals
the same request proved alone and the oracle's proof of it, under overlap and
under key eviction."""
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def keys():
    out = []
    for i, nc in enumerate((150, 700, 2500)):
        sc = S.SynthCircuit(40 + i, nc, 24, 4)
        out.append((sc, sc.zkey(90 + i)))
    return out


def blinders(j):
    rng = random.Random(j)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


def alone(backend, zk, w, r, s):
    c = backend.prepare(S.ProvingKey.from_bytes(zk))
    p = c.prove_with_blinders(w, r, s)
    c.close()
    return p


@pytest.mark.parametrize("lanes,budget,max_batch", [(4, 0, 64), (3, 1, 64), (2, 0, 1)])
def test_served_results_equal_proofs_alone(backend, keys, lanes, budget, max_batch):
    # budget 1: every new key evicts the idle ones (LRU path); max_batch 1: plain serving
    srv = S.ProofServer(backend, budget, lanes, max_batch)
    for i, (_, zk) in enumerate(keys):
        srv.register_key(i, zk)
    rng = random.Random(lanes)
    jobs = []
    for j in range(18):
        i = rng.randrange(len(keys))
        w = keys[i][0].witness(j)
        r, s = blinders(j)
        jobs.append((srv.submit(i, w, r, s), i, w, r, s))
    got = [(srv.wait(t)[0], i, w, r, s) for t, i, w, r, s in jobs]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(jobs)
    if budget:
        assert st["evicted"] > 0
    oks = [O.Zkey(zk) for _, zk in keys]
    for p, i, w, r, s in got:
        assert p == alone(backend, keys[i][1], w, r, s)
        ok = oks[i]
        assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        assert ok.verify(w[32:32 * (1 + ok.n_public)], p.to_bytes())


def test_server_errors(backend, keys):
    srv = S.ProofServer(backend, 0, 2)
    srv.register_key(0, keys[0][1])
    with pytest.raises(S.InvalidArgumentError):
        srv.submit(7, keys[0][0].witness(1), *blinders(1))
    t = srv.submit(0, keys[0][0].witness(1)[:-32], *blinders(1))
    with pytest.raises(S.WitnessLengthError):
        srv.wait(t)
    srv.close()
