"""Device faults without a GPU fault: a CUDA status injected on the host makes
the next entry point fail as the driver's would; a sticky one puts the backend
out of use (every later call refused before any CUDA call), a non-sticky one
does not.  And a key that does not fit with its window tables is prepared as a
compact key (plain bases, one bucket set per window) whose proofs equal the
oracle's (crates/cuda/src/context.rs:134-215; msm.rs:966,1117)."""
import os
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu

LAUNCH_FAILURE, MEMORY_ALLOCATION, ECC_UNCORRECTABLE = 719, 2, 214


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


@pytest.fixture(scope="module")
def small():
    sc = S.SynthCircuit(seed=901, n_constraints=2000, n_inputs=32, n_public=4)
    zk = sc.zkey(902)
    ok = O.Zkey(zk)
    yield sc, zk, ok
    ok.close()


def test_injected_faults(small):
    sc, zk, ok = small
    b = S.CudaBackend(0)
    c = b.prepare(S.ProvingKey.from_bytes(zk))
    w = sc.witness(5)
    r, s = blinders(5)
    good = c.prove_with_blinders(w, r, s)
    # out of memory: DEVICE_MEMORY, nothing sticks
    b.inject_fault(MEMORY_ALLOCATION)
    with pytest.raises(S.DeviceMemoryError):
        c.prove_with_blinders(w, r, s)
    assert b.fault() == 0
    assert c.prove_with_blinders(w, r, s) == good
    # a device fault the context survives
    b.inject_fault(ECC_UNCORRECTABLE)
    with pytest.raises(S.DeviceError):
        b.prove_batch([(c, w, r, s)])
    assert b.fault() == 0
    assert b.prove_batch([(c, w, r, s)]) == [good]
    # sticky: this call and every later one on the backend refused, no kernel launched
    b.inject_fault(LAUNCH_FAILURE)
    with pytest.raises(S.DeviceError, match="sticky"):
        c.prove_with_blinders(w, r, s)
    assert b.fault() == LAUNCH_FAILURE
    launches = S.launch_count()
    for call in (lambda: c.prove_with_blinders(w, r, s), lambda: b.prove_batch([(c, w, r, s)]),
                 lambda: b.prepare(S.ProvingKey.from_bytes(zk)),
                 lambda: S.CudaMsm(b).msm_g1(bytes(64 * 4), bytes(32 * 4))):
        with pytest.raises(S.DeviceError, match="out of use"):
            call()
    assert S.launch_count() == launches
    c.close()
    b.close()
    # the injection took this backend alone; another one proves as before
    b2 = S.CudaBackend(0)
    c2 = b2.prepare(S.ProvingKey.from_bytes(zk))
    assert b2.fault() == 0
    assert c2.prove_with_blinders(w, r, s) == good
    c2.close()
    b2.close()


def test_compact_key_when_tables_do_not_fit(small):
    sc, zk, ok = small
    pk = S.ProvingKey.from_bytes(zk)
    full = pk.plan(1 << 40)
    assert full["window_tables"] == 1
    b = S.CudaBackend(0, vram_limit=full["key_bytes"] + full["workspace_bytes"] - 1)
    c = b.prepare(pk)
    assert not c.window_tables()
    assert c.device_bytes() < full["key_bytes"]
    jobs = []
    for k in range(3):
        w = sc.witness(40 + k)
        r, s = blinders(40 + k)
        p = c.prove_with_blinders(w, r, s)
        assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        jobs.append((c, w, r, s, p))
    # batched submissions of a compact key run on host lanes, same proofs
    assert b.prove_batch([j[:4] for j in jobs]) == [j[4] for j in jobs]
    # another window width at run time (no tables to rebuild)
    t = c.tuning()
    c.set_tuning(t["msm_window_bits_witness"] + 2, t["msm_window_bits_h"] + 1, t["ntt_tile_log"], t["ntt_outer_log_l"])
    assert c.prove_with_blinders(*jobs[0][1:4]) == jobs[0][4]
    c.close()
    b.close()


def test_compact_key_by_environment_matches_oracle():
    sc = S.SynthCircuit(seed=903, n_constraints=21000, n_inputs=200, n_public=9)
    zk = sc.zkey(904)
    ok = O.Zkey(zk)
    os.environ["G16_CUDA_WINDOW_TABLES"] = "0"
    try:
        b = S.CudaBackend(0)
        c = b.prepare(S.ProvingKey.from_bytes(zk))
    finally:
        del os.environ["G16_CUDA_WINDOW_TABLES"]
    assert not c.window_tables()
    w = sc.witness(9)
    r, s = blinders(9)
    p = c.prove_with_blinders(w, r, s)
    assert p.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
    assert ok.verify(w[32:32 * (1 + ok.n_public)], p.to_bytes())
    c.close()
    b.close()
    ok.close()


def test_batch_mixing_compact_and_table_keys(small, backend):
    """A submission with a compact key runs on host lanes; every proof equals its single proof."""
    sc, zk, ok = small
    os.environ["G16_CUDA_WINDOW_TABLES"] = "0"
    try:
        compact = backend.prepare(S.ProvingKey.from_bytes(zk))
    finally:
        del os.environ["G16_CUDA_WINDOW_TABLES"]
    tables = backend.prepare(S.ProvingKey.from_bytes(zk))
    assert not compact.window_tables() and tables.window_tables()
    jobs = []
    for k, c in enumerate([tables, compact, tables, compact]):
        w = sc.witness(70 + k)
        r, s = blinders(70 + k)
        jobs.append((c, w, r, s))
    singles = [c.prove_with_blinders(w, r, s) for c, w, r, s in jobs]
    assert backend.prove_batch(jobs) == singles
    # the same key held both ways gives the same proof
    assert compact.prove_with_blinders(*jobs[0][1:]) == singles[0]
    compact.close()
    tables.close()
