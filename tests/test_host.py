"""CPU-side checks of the product library: it loads, exports every symbol the
public header declares, refuses to compute without a GPU, and its host code
(format readers/writers, the synthetic generator) agrees with the oracle."""
import os
import re

import pytest

import oracle as O
import snarkrs_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "g16b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(g16_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) > 30
    lib = S.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_no_cpu_fallback_without_a_device():
    with pytest.raises(S.DeviceError):
        S.CudaBackend(0)


@pytest.fixture(scope="module")
def small():
    sc = S.SynthCircuit(seed=11, n_constraints=300, n_inputs=24, n_public=5)
    return sc, sc.zkey(1234), sc.witness(77)


def test_synth_key_proves_and_verifies_under_the_oracle(small):
    sc, zk, w = small
    ok = O.Zkey(zk)
    assert (ok.n_vars, ok.n_public, ok.domain_size) == (sc.n_vars, 5, sc.domain_size)
    proof = ok.prove(w, O.to_mont(5), O.to_mont(7))
    pub = w[32:32 * (1 + ok.n_public)]
    assert ok.verify(pub, proof)
    bad = bytearray(pub)
    bad[1] ^= 1
    assert not ok.verify(bytes(bad), proof)


def test_domain_rule_matches_snarkjs(small):
    """domain = 2^(floor(log2(nConstraints + nPublic)) + 1) (setup.rs:125-134)."""
    for nc, npub, want in ((300, 5, 512), (2 ** 15, 16, 2 ** 16), (1000, 24, 2048), (1008, 16, 2048), (1007, 16, 1024)):
        sc = S.SynthCircuit(seed=1, n_constraints=nc, n_inputs=max(npub, 20), n_public=npub)
        assert sc.domain_size == want, (nc, npub)


def test_witness_value_distribution():
    sc = S.SynthCircuit(seed=3, n_constraints=4000, n_inputs=256, n_public=16)
    w = sc.witness(9)
    vals = [S.fr_from_mont_bytes(w[32 * i:32 * i + 32]) for i in range(sc.n_vars)]
    frac01 = sum(v in (0, 1) for v in vals) / len(vals)
    small = sum(1 < v < 2 ** 32 for v in vals) / len(vals)
    assert 0.5 < frac01 < 0.68 and 0.15 < small < 0.25
    assert vals[0] == 1
    # different witness seeds share the structure: 0/1/small wires agree, inputs differ
    w2 = sc.witness(10)
    assert w2[32:64] != w[32:64]


def test_zkey_reader_agrees_with_oracle_reader(small):
    sc, zk, _ = small
    pk = S.ProvingKey.from_bytes(zk)
    ok = O.Zkey(zk)
    assert (pk.n_vars, pk.n_public, pk.domain_size) == (ok.n_vars, ok.n_public, ok.domain_size)
    assert len(pk.ic) == pk.n_public + 1
    assert O.g1_on_curve(pk.alpha_g1) and O.g2_on_curve(pk.delta_g2)


def test_zkey_reader_refuses_malformed(small):
    _, zk, _ = small
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_bytes(b"nope" + zk[4:])
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_bytes(zk[: len(zk) // 2])
    # a header point coordinate at or above q
    bad = bytearray(zk)
    i = zk.find((O.Q_MOD).to_bytes(32, "little"))     # section 2 stores q itself
    assert i > 0
    hdr = i + 32 + 4 + 32 + 12                          # alpha_g1.x
    bad[hdr:hdr + 32] = (O.Q_MOD).to_bytes(32, "little")
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_bytes(bytes(bad))


def test_wtns_round_trip_and_constant_wire(small):
    _, _, w = small
    assert S.load_witness(S.write_witness(w)) == w
    bad = bytearray(w)
    bad[:32] = bytes(32)
    with pytest.raises(S.FormatError):
        S.load_witness(S.write_witness(bytes(bad)))


def test_r1cs_writer_layout(small):
    sc, _, _ = small
    r = sc.r1cs()
    assert r[:4] == b"r1cs"
    hdr = r.find(O.R_MOD.to_bytes(32, "little"))
    n_wires, n_out, n_pub, n_prv = (int.from_bytes(r[hdr + 32 + 4 * i:hdr + 36 + 4 * i], "little") for i in range(4))
    assert (n_wires, n_out, n_pub, n_prv) == (sc.n_vars, 0, 5, 19)


# cudaError_t values from the CUDA runtime's driver_types.h, each with the
# classes the reference's is_device_fault / is_sticky give its CUresult twin
# (crates/cuda/src/context.rs:146-215); 0 for calls rejected every time.
CUDA_STATUS_CLASSES = {
    0: 0,      # cudaSuccess
    1: 0,      # cudaErrorInvalidValue
    2: 1,      # cudaErrorMemoryAllocation
    46: 1,     # cudaErrorDevicesUnavailable
    98: 0,     # cudaErrorInvalidDeviceFunction
    100: 0,    # cudaErrorNoDevice
    214: 1,    # cudaErrorECCUncorrectable
    220: 1,    # cudaErrorNvlinkUncorrectable
    226: 3,    # cudaErrorContained
    400: 0,    # cudaErrorInvalidResourceHandle
    600: 0,    # cudaErrorNotReady
    700: 3,    # cudaErrorIllegalAddress
    701: 0,    # cudaErrorLaunchOutOfResources
    702: 3,    # cudaErrorLaunchTimeout
    710: 3,    # cudaErrorAssert
    714: 3,    # cudaErrorHardwareStackError
    715: 3,    # cudaErrorIllegalInstruction
    716: 3,    # cudaErrorMisalignedAddress
    717: 3,    # cudaErrorInvalidAddressSpace
    718: 3,    # cudaErrorInvalidPc
    719: 3,    # cudaErrorLaunchFailure
    802: 1,    # cudaErrorSystemNotReady
    805: 1, 806: 1, 807: 1, 808: 1, 809: 1, 810: 1,   # MPS failures
    900: 0,    # cudaErrorStreamCaptureUnsupported
    909: 1,    # cudaErrorTimeout
    911: 1,    # cudaErrorExternalDevice
    999: 1,    # cudaErrorUnknown
}


def test_cuda_status_classes():
    got = {code: S.cuda_error_class(code) for code in CUDA_STATUS_CLASSES}
    assert got == CUDA_STATUS_CLASSES
    assert S.FAULT_DEVICE == 1 and S.FAULT_STICKY == 2


def test_key_plan_falls_back_to_a_compact_key(monkeypatch):
    # large enough that the compact key and its workspace are the smaller plan
    sc = S.SynthCircuit(seed=901, n_constraints=3000, n_inputs=24, n_public=5)
    pk = S.ProvingKey.from_bytes(sc.zkey(902))
    full = pk.plan(1 << 40)
    assert full["window_tables"] == 1
    need_full = full["key_bytes"] + full["workspace_bytes"]
    compact = pk.plan(need_full - 1)
    assert compact["window_tables"] == 0
    assert compact["key_bytes"] < full["key_bytes"]
    assert 8 <= compact["msm_window_bits_witness"] <= 20 and 8 <= compact["msm_window_bits_h"] <= 20
    assert pk.plan(compact["key_bytes"] + compact["workspace_bytes"])["window_tables"] == 0
    with pytest.raises(S.DeviceMemoryError, match="compact key"):
        pk.plan(compact["key_bytes"] + compact["workspace_bytes"] - 1)
    monkeypatch.setenv("G16_CUDA_WINDOW_TABLES", "0")
    assert pk.plan(1 << 40)["window_tables"] == 0


def test_compact_key_is_much_smaller():
    sc = S.SynthCircuit(seed=5, n_constraints=1 << 14, n_inputs=64, n_public=4)
    pk = S.ProvingKey.from_bytes(sc.zkey(6))
    full = pk.plan(1 << 50)
    compact = pk.plan(full["key_bytes"] + full["workspace_bytes"] - 1)
    assert compact["key_bytes"] * 8 < full["key_bytes"]


def test_readiness_entry_points_refuse_null_handles():
    # g16_batch_reserve and g16_circuit_warm check their handles before any CUDA call
    with pytest.raises(S.InvalidArgumentError):
        S.check(S.lib().g16_batch_reserve(None, 0, None))
    with pytest.raises(S.InvalidArgumentError):
        S.check(S.lib().g16_circuit_warm(None, 2))


def _zkey_sections(zk):
    import struct
    out, off = {}, 12
    while off + 12 <= len(zk):
        sid, size = struct.unpack_from("<IQ", zk, off)
        out[sid] = (off + 12, size)
        off += 12 + size
    return out


def test_query_point_checks_follow_load_and_load_unchecked(small):
    # ProvingKey::load checks every query point on its curve; load_unchecked does not
    # (formats/src/lib.rs:430-505): a corrupted A-query point is refused only by the first
    _, zk, _ = small
    start, size = _zkey_sections(zk)[5]            # section 5: the A query, packed G1
    bad = bytearray(zk)
    for i in range(0, size, 64):                   # the first finite point
        if any(bad[start + i:start + i + 64]):
            bad[start + i + 40] ^= 0x01            # its y, one bit off: off the curve
            break
    else:
        pytest.skip("no finite A-query point")
    with pytest.raises(S.FormatError):
        S.ProvingKey.from_bytes(bytes(bad), check_points=True)
    S.ProvingKey.from_bytes(bytes(bad), check_points=False).close()
