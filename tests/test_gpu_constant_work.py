"""Constant-work MSMs (the reference's Work::Constant, crates/msm/src/lib.rs:206-220;
CudaBackend::constant_work, crates/cuda/src/backend.rs:100-118): results are the
variable-work results bit for bit, and the work no longer depends on the witness."""
import random

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD))), O.to_bytes(O.to_mont(rng.randrange(1, O.R_MOD)))


def madds(fn):
    """Mixed additions the accumulate kernels performed during fn()."""
    S.kernel_timing_reset()
    S.kernel_timing(True)
    try:
        out = fn()
    finally:
        S.kernel_timing(False)
    rep = S.kernel_timing_report()
    return out, sum(v[2] for k, v in rep.items() if k.startswith("msm_accumulate"))


def test_constant_work_proofs_equal_and_work_follows_the_key(backend):
    sc = S.SynthCircuit(seed=61, n_constraints=3000, n_inputs=40, n_public=5)
    zk = sc.zkey(515)
    ok = O.Zkey(zk)
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    w1, w2 = sc.witness(1), sc.witness(2)
    # a sparse witness: every private input wire zero where the circuit allows it is
    # not needed; two seeds already differ in their zero / one counts
    r, s = blinders(1)
    try:
        v1, m_var1 = madds(lambda: circ.prove_with_blinders(w1, r, s))
        v2, m_var2 = madds(lambda: circ.prove_with_blinders(w2, r, s))
        backend.set_constant_work(True)
        c1, m_cw1 = madds(lambda: circ.prove_with_blinders(w1, r, s))
        c2, m_cw2 = madds(lambda: circ.prove_with_blinders(w2, r, s))
        c1b = circ.prove_with_blinders(w1, r, s)        # graph replay in constant mode
    finally:
        backend.set_constant_work(False)
    assert c1 == v1 == c1b and c2 == v2
    assert c1.to_bytes() == ok.prove(w1, O.from_bytes(r), O.from_bytes(s))
    # variable work follows the witness; constant work does not, and does more
    assert m_var1 != m_var2
    assert m_cw1 == m_cw2 > max(m_var1, m_var2)
    # back in variable mode the graph captured there is used again
    assert circ.prove_with_blinders(w1, r, s) == v1
    circ.close()


@pytest.mark.parametrize("g2", [False, True])
def test_constant_work_msm_matches_oracle(backend, g2):
    n = 3000
    bases = S.synth_points(2 if g2 else 1, 17, n)
    scal = bytearray(S.synth_scalars(18, n, 1))          # 70% zeros and ones
    scal[32 * 5:32 * 6] = bytes(32)
    msm = S.CudaMsm(backend)
    fn = msm.msm_g2 if g2 else msm.msm_g1
    want = (O.msm_g2 if g2 else O.msm_g1)(bases, bytes(scal))
    backend.set_constant_work(True)
    try:
        assert fn(bases, bytes(scal)) == want
        assert fn(bases, bytes(32 * n)) == (bytes(128) if g2 else bytes(64))   # all-zero scalars: infinity
    finally:
        backend.set_constant_work(False)
