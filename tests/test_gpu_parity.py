"""GPU parity: every CUDA result through the C ABI is bit-identical to the
oracle (the CPU restatement of the reference prover) on the same seeded
inputs; full sizes are covered through size-independent properties."""
import random

import pytest

import oracle as O
import pyref as P
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu

R = O.R_MOD


def rand_mont(n, seed):
    rng = random.Random(seed)
    return b"".join(O.to_bytes(O.to_mont(rng.randrange(R))) for _ in range(n))


# ------------------------------------------------------------------ NTT
@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8, 10, 11, 12, 13, 16, 18])
def test_ntt_all_modes_match_oracle(backend, log_n):
    ntt = S.CudaNtt(backend)
    data = rand_mont(1 << log_n, log_n)
    assert ntt.ntt(data) == O.ntt(log_n, O.NTT_FORWARD, data)
    assert ntt.ntt(data, inverse=True) == O.ntt(log_n, O.NTT_INVERSE, data)
    assert ntt.intt_coset_ntt(data) == O.ntt(log_n, O.NTT_INTT_COSET_NTT, data)
    assert ntt.coset_ntt(data) == O.ntt(log_n, O.NTT_COSET_FORWARD, data)
    shift = O.to_mont(7)
    assert ntt.coset_ntt(data, O.to_bytes(shift), inverse=True) == O.ntt(log_n, O.NTT_COSET_INVERSE, data, shift)


@pytest.mark.parametrize("log_n", [20, 22, 24])
def test_ntt_config_sizes_all_modes_match_oracle(backend, log_n):
    """Every transform of the standalone-kernel configuration (log n = 20, 22, 24):
    forward, inverse (with 1/n), coset forward with the proving shift, coset inverse
    with another shift, and intt_coset_ntt, each against the oracle."""
    ntt = S.CudaNtt(backend)
    data = S.synth_scalars(log_n, 1 << log_n, 0)          # standard-form values are valid Montgomery limbs
    assert ntt.ntt(data) == O.ntt(log_n, O.NTT_FORWARD, data)
    assert ntt.ntt(data, inverse=True) == O.ntt(log_n, O.NTT_INVERSE, data)
    assert ntt.coset_ntt(data) == O.ntt(log_n, O.NTT_COSET_FORWARD, data)
    shift = O.to_mont(5)
    assert ntt.coset_ntt(data, O.to_bytes(shift), inverse=True) == O.ntt(log_n, O.NTT_COSET_INVERSE, data, shift)
    assert ntt.intt_coset_ntt(data) == O.ntt(log_n, O.NTT_INTT_COSET_NTT, data)


def _limb_sum(data, sign=None):
    """sum_i s_i x_i mod r over 32-byte little-endian values, via 32-bit limb sums in numpy."""
    import numpy as np
    a = np.frombuffer(data, dtype=np.uint32).reshape(-1, 8).astype(np.int64)
    if sign is not None:
        a = a * sign[:, None]
    return sum(int(a[:, k].sum()) << (32 * k) for k in range(8)) % R


def test_ntt_2_24_round_trip_and_sums(backend):
    """2^24: inverse(forward(x)) = x; forward(x)[0] = sum x_i and forward(x)[n/2] = sum (-1)^i x_i."""
    import numpy as np
    log_n = 24
    n = 1 << log_n
    ntt = S.CudaNtt(backend)
    x = S.synth_scalars(101, n, 0)
    fx = ntt.ntt(x)
    assert ntt.ntt(fx, inverse=True) == x
    # Montgomery limbs are linear, so the identities hold on the raw limbs mod r
    assert O.from_bytes(fx[:32]) == _limb_sum(x)
    alt = np.where(np.arange(n) % 2 == 0, 1, -1).astype(np.int64)
    assert O.from_bytes(fx[32 * (n // 2):32 * (n // 2) + 32]) == _limb_sum(x, alt)


# ------------------------------------------------------------------ MSM
def msm_pair(backend, n, dist, seed, g2=False):
    bases = S.synth_points(2 if g2 else 1, seed, n)
    scal = S.synth_scalars(seed + 1, n, dist)
    msm = S.CudaMsm(backend)
    got = (msm.msm_g2 if g2 else msm.msm_g1)(bases, scal)
    want = (O.msm_g2 if g2 else O.msm_g1)(bases, scal)
    return got, want


@pytest.mark.parametrize("n", [1, 2, 3, 31, 100, 1000, 4096])
@pytest.mark.parametrize("dist", [0, 1])
def test_msm_g1_small_matches_oracle(backend, n, dist):
    got, want = msm_pair(backend, n, dist, 1000 + n)
    assert got == want


@pytest.mark.parametrize("n,dist", [(1 << 16, 0), (1 << 16, 1), (1 << 20, 0), (1 << 20, 1)])
def test_msm_g1_config_sizes_match_oracle(backend, n, dist):
    got, want = msm_pair(backend, n, dist, 7 * n + dist)
    assert got == want


def test_msm_g1_2_22_matches_oracle_and_splits(backend):
    """The largest configured G1 MSM (2^22 points): equal to the oracle for both scalar
    distributions, and to the sum of the MSMs of its two halves."""
    n = 1 << 22
    bases = S.synth_points(1, 4242, n)
    msm = S.CudaMsm(backend)
    for dist in (0, 1):
        scal = S.synth_scalars(4243 + dist, n, dist)
        got = msm.msm_g1(bases, scal)
        assert got == O.msm_g1(bases, scal)
        h = n // 2
        lo = msm.msm_g1(bases[:64 * h], scal[:32 * h])
        hi = msm.msm_g1(bases[64 * h:], scal[32 * h:])
        assert O.g1_add(lo, hi) == got


@pytest.mark.parametrize("n,dist", [(1, 0), (77, 0), (4096, 1), (1 << 16, 0)])
def test_msm_g2_matches_oracle(backend, n, dist):
    got, want = msm_pair(backend, n, dist, 31 + n, g2=True)
    assert got == want


@pytest.mark.parametrize("dist", [0, 1])
def test_msm_g2_2_20(backend, dist):
    """The configured G2 MSM, 2^20 points, uniform scalars and 70% in {0,1}."""
    got, want = msm_pair(backend, 1 << 20, dist, 9 + dist, g2=True)
    assert got == want


def test_msm_edge_cases(backend):
    """Zeros, ones, r-1, infinity bases, repeated bases (P+P in a bucket), opposite bases (P-P)."""
    rng = random.Random(12)
    pts = [P.pt_mul(P.G1, rng.randrange(1, R)) for _ in range(40)]
    pts[3] = None
    pts[5] = pts[4]
    pts[7] = P.pt_neg(pts[6])
    pts[9] = pts[8]
    ks = [rng.randrange(R) for _ in pts]
    ks[0], ks[1], ks[2] = 0, 1, R - 1
    ks[5] = ks[4]                  # same bucket, same point: doubling inside a bucket
    ks[7] = ks[6]                  # P and -P with the same scalar cancel
    ks[9] = (R - ks[8]) % R        # P with k and P with -k cancel
    bases = b"".join(P.pack_g1(p) for p in pts)
    scal = b"".join(k.to_bytes(32, "little") for k in ks)
    msm = S.CudaMsm(backend)
    assert msm.msm_g1(bases, scal) == O.msm_g1(bases, scal) == P.pack_g1(P.msm_naive(pts, ks))
    # all zero scalars and all infinity bases give infinity
    assert msm.msm_g1(bases, bytes(32 * len(pts))) == bytes(64)
    assert msm.msm_g1(bytes(64 * 8), scal[:32 * 8]) == bytes(64)
    # Montgomery-form scalars give the same result
    mont = b"".join(O.to_bytes(O.to_mont(k)) for k in ks)
    assert msm.msm_g1(bases, mont, S.SCALARS_MONTGOMERY) == O.msm_g1(bases, scal)
    # fat buckets: one repeated scalar over many points
    n = 5000
    bases = S.synth_points(1, 5, n)
    k = (rng.randrange(R)).to_bytes(32, "little")
    assert msm.msm_g1(bases, k * n) == O.msm_g1(bases, k * n)
    with pytest.raises(S.BackendError):
        msm.msm_g1(bases[:64 * 10], k * 11)


def test_msm_repeatable(backend):
    """Repeated and interleaved MSMs are bit-identical (stale scratch must not leak)."""
    msm = S.CudaMsm(backend)
    b1, s1 = S.synth_points(1, 1, 3000), S.synth_scalars(2, 3000, 0)
    b2, s2 = S.synth_points(1, 3, 100), S.synth_scalars(4, 100, 1)
    r1 = msm.msm_g1(b1, s1)
    msm.msm_g1(b2, s2)
    assert msm.msm_g1(b1, s1) == r1


# ------------------------------------------------------------------ prover
@pytest.fixture(scope="module")
def circuits():
    out = {}
    for name, nc, ni, npub in (("tiny", 200, 20, 4), ("small", 3000, 64, 8), ("config0", 1 << 15, 256, 16)):
        sc = S.SynthCircuit(seed=sum(map(ord, name)), n_constraints=nc, n_inputs=ni, n_public=npub)
        zk = sc.zkey(4242)
        out[name] = (sc, zk, O.Zkey(zk))
    return out


def blinders(seed):
    rng = random.Random(seed)
    return O.to_bytes(O.to_mont(rng.randrange(1, R))), O.to_bytes(O.to_mont(rng.randrange(1, R)))


@pytest.mark.parametrize("name", ["tiny", "small", "config0"])
def test_proof_bit_exact_and_verifies(backend, circuits, name):
    sc, zk, ok = circuits[name]
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    for ws in (1, 2):
        w = sc.witness(ws)
        r, s = blinders(ws)
        proof = circ.prove_with_blinders(w, r, s)
        want = ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        assert proof.to_bytes() == want
        assert ok.verify(w[32:32 * (1 + ok.n_public)], proof.to_bytes())
    circ.close()


def test_stages_match_oracle(backend, circuits):
    sc, zk, ok = circuits["small"]
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    w = sc.witness(3)
    h = circ.compute_h(w)
    h_host = circ.h_to_host(h)
    assert h_host == ok.compute_h(w)
    m = circ.msms(w, h)
    want = ok.msms(w, h_host)
    assert m.as_dict() == want
    assert circ.h_and_msms(w).as_dict() == want


def test_trace_blinders_and_repeatability(backend, circuits):
    """Fixed blinders TRACE_R/TRACE_S (crates/groth16/src/trace.rs:43-47); proofs repeat bit for bit."""
    sc, zk, ok = circuits["small"]
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    other = backend.prepare(S.ProvingKey.from_bytes(circuits["tiny"][1]))
    r, s = O.to_bytes(O.to_mont(0x57726F6E67205231)), O.to_bytes(O.to_mont(0x57726F6E67205332))
    w = sc.witness(5)
    p1 = circ.prove_with_blinders(w, r, s)
    other.prove_with_blinders(circuits["tiny"][0].witness(1), r, s)       # dirty the device in between
    p2 = circ.prove_with_blinders(w, r, s)
    assert p1 == p2
    assert p1.to_bytes() == ok.prove(w, O.from_bytes(r), O.from_bytes(s))


def test_prove_errors(backend, circuits):
    sc, zk, _ = circuits["tiny"]
    circ = backend.prepare(S.ProvingKey.from_bytes(zk))
    w = sc.witness(1)
    r, s = blinders(1)
    with pytest.raises(S.WitnessLengthError):
        circ.prove_with_blinders(w[:-32], r, s)
    bad = bytearray(w)
    bad[:32] = bytes(32)
    with pytest.raises(S.ConstantWireError):
        circ.prove_with_blinders(bytes(bad), r, s)
    other = backend.prepare(S.ProvingKey.from_bytes(circuits["small"][1]))
    h = other.compute_h(circuits["small"][0].witness(1))
    with pytest.raises(S.BackendError):
        circ.msms(w, h)
    tight = S.CudaBackend(0, vram_limit=1)
    with pytest.raises(S.DeviceMemoryError):
        tight.prepare(S.ProvingKey.from_bytes(zk))
    tight.close()


def test_batch_equals_singles(backend, circuits):
    jobs = []
    circs = {}
    for name in ("tiny", "small"):
        sc, zk, _ = circuits[name]
        circs[name] = backend.prepare(S.ProvingKey.from_bytes(zk))
        for ws in range(3):
            r, s = blinders(100 + ws)
            jobs.append((circs[name], sc.witness(ws), r, s))
    batch = backend.prove_batch(jobs)
    oks = {name: circuits[name][2] for name in circs}
    names = [name for name in ("tiny", "small") for _ in range(3)]
    for (c, w, r, s), p, name in zip(jobs, batch, names):
        assert p == c.prove_with_blinders(w, r, s)
        assert p.to_bytes() == oks[name].prove(w, O.from_bytes(r), O.from_bytes(s))


def test_device_key_generation_is_the_host_one(backend):
    """g16_synth_zkey_device: the point sections computed on the GPU give the same
    .zkey bytes as the host generator (and so the same proofs)."""
    for nc, npub in ((300, 4), (20000, 16)):
        host = S.SynthCircuit(seed=808 + nc, n_constraints=nc, n_inputs=40, n_public=npub).zkey(99)
        dev = S.SynthCircuit(seed=808 + nc, n_constraints=nc, n_inputs=40, n_public=npub).zkey(99, device=0)
        assert dev == host


def test_live_sets_with_every_base_at_infinity(backend, circuits):
    """The witness MSMs skip wires whose base is the point at infinity (the reference's
    prescan and key_live).  With every B query base at infinity the B live set is empty:
    B1 and B2 come out at infinity and the A, L and H outputs are those of the intact key;
    with every A base at infinity as well, A is at infinity too."""
    import ctypes
    sc, zk, ok = circuits["small"]
    w = sc.witness(4)
    intact = backend.prepare(S.ProvingKey.from_bytes(zk)).h_and_msms(w).as_dict()
    assert intact == ok.msms(w, ok.compute_h(w))
    pk = S.ProvingKey.from_bytes(zk)
    nv = pk.n_vars
    ctypes.memset(ctypes.addressof(pk._view.b_g1_query.contents), 0, 64 * nv)
    ctypes.memset(ctypes.addressof(pk._view.b_g2_query.contents), 0, 128 * nv)
    circ = backend.prepare(pk)
    got = circ.h_and_msms(w).as_dict()
    assert got["b_g1"] == bytes(64) and got["b_g2"] == bytes(128)
    assert all(got[k] == intact[k] for k in ("a_g1", "l_g1", "h_g1"))
    circ.close()
    ctypes.memset(ctypes.addressof(pk._view.a_query.contents), 0, 64 * nv)
    circ = backend.prepare(pk)
    got = circ.h_and_msms(w).as_dict()
    assert got["a_g1"] == bytes(64) and got["b_g1"] == bytes(64)
    assert got["l_g1"] == intact["l_g1"] and got["h_g1"] == intact["h_g1"]
    circ.close()
