"""Bit-exact parity at the benchmarked configuration: the plain prove of the
seeded 1,100,000-constraint circuit (domain 2^21, 1,100,257 wires), the
workload bench.py times.  The CUDA proof must equal the oracle's proof of the
same witness with the same r and s, byte for byte, and pass the pairing check
(the reference's CUDA-vs-CPU identity at equal blinders,
crates/cuda/tests/size_sweep_gpu.rs:140-200).  Two witnesses are proved: the
first runs the enqueue path, the second replays the workspace's captured CUDA
graph, the path the timed region uses."""
import pytest

import bench
import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def headline():
    sc = S.SynthCircuit(bench.CIRCUIT_SEED, bench.N_CONSTRAINTS, bench.N_INPUTS, bench.N_PUBLIC)
    zk = bench.synth_key(sc, bench.N_CONSTRAINTS)
    ok = O.Zkey(zk)
    yield sc, zk, ok
    ok.close()


def test_headline_prove_bit_exact_against_the_oracle(backend, headline):
    sc, zk, ok = headline
    assert sc.domain_size == 1 << 21
    circ = backend.prepare(S.ProvingKey.from_bytes(zk, check_points=False))
    try:
        for step in (0, 1):
            seed = bench.witness_seed(0, step)
            w = sc.witness(seed)
            r, s = bench.blinders(seed)
            got = circ.prove_with_blinders(w, r, s).to_bytes()
            want = ok.prove(w, O.from_bytes(r), O.from_bytes(s))
            assert got == want, "step %d: CUDA proof differs from the oracle's" % step
            assert ok.verify(w[32:32 * (1 + ok.n_public)], got)
    finally:
        circ.close()


def test_headline_stages_match_the_oracle(backend, headline):
    """H and the five MSM outputs separately, so that a mismatch names its stage."""
    sc, zk, ok = headline
    circ = backend.prepare(S.ProvingKey.from_bytes(zk, check_points=False))
    try:
        w = sc.witness(bench.witness_seed(0, 7))
        h = circ.compute_h(w)
        h_host = circ.h_to_host(h)
        assert h_host == ok.compute_h(w)
        assert circ.msms(w, h).as_dict() == ok.msms(w, h_host)
    finally:
        circ.close()
