"""snarkrs_b200: B200-native Groth16 / BN254 proving hot path.

A Python mirror of the reference's backend interface for the prove path
(zemse/snarkrs ``crates/groth16/src/lib.rs:371-455`` Backend /
PreparedCircuit, ``crates/msm/src/lib.rs:52-82`` MsmBackend,
``crates/ntt/src/lib.rs:415-584`` the NTT API), bound through ctypes to the
C ABI in ``include/g16b200.h`` implemented by ``libg16b200.so`` (hand-written
sm_100a CUDA).  There is no CPU fallback: every compute call runs on the GPU
or raises.

Byte conventions follow the reference's packed layout: field elements are 32
little-endian bytes in Montgomery form (the in-memory bits of an arkworks
``Fr``), MSM scalars may be standard or Montgomery form, G1 points are 64
bytes, G2 points 128 bytes, the point at infinity is all-zero.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libg16b200.so")

G16_OK = 0
SCALARS_STANDARD, SCALARS_MONTGOMERY = 0, 1
NTT_FORWARD, NTT_INVERSE, NTT_INTT_COSET_NTT, NTT_COSET_FORWARD, NTT_COSET_INVERSE = range(5)

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583


# ---- errors: ProveError (crates/groth16/src/lib.rs:81-154) ----
class ProveError(Exception):
    code = -1


class WitnessLengthError(ProveError):
    code = 1


class ConstantWireError(ProveError):
    code = 2


class BackendError(ProveError):
    code = 3


class DeviceError(ProveError):
    code = 4


class DeviceMemoryError(ProveError):
    code = 5


class SelfVerifyError(ProveError):
    code = 6


class TimeoutError_(ProveError):
    code = 7


class InvalidArgumentError(ProveError):
    code = 8


class FormatError(ProveError):
    """ZkeyError: malformed .zkey / .wtns bytes."""
    code = 9


class VerifyError(ProveError):
    """verify::VerifyError (crates/groth16/src/verify.rs:17-33): the proof does not verify."""
    code = 10


_ERRORS = {c.code: c for c in (WitnessLengthError, ConstantWireError, BackendError, DeviceError,
                                DeviceMemoryError, SelfVerifyError, TimeoutError_, InvalidArgumentError,
                                FormatError, VerifyError)}

_lib = None


def lib():
    """Load libg16b200.so; raise if it is missing (no fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libg16b200.so is not built; run `python -m snarkrs_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.g16_last_error.restype = ctypes.c_size_t
        L.g16_backend_name.restype = ctypes.c_char_p
        L.g16_backend_vram_used.restype = ctypes.c_uint64
        L.g16_backend_free.argtypes = [vp]
        L.g16_zkey_free.argtypes = [vp]
        L.g16_circuit_free.argtypes = [vp]
        L.g16_hpoly_free.argtypes = [vp]
        L.g16_synth_free.argtypes = [vp]
        L.g16_server_free.argtypes = [vp]
        for f in ("g16_circuit_n_vars", "g16_circuit_n_public", "g16_circuit_domain_size",
                  "g16_synth_n_vars", "g16_synth_domain_size"):
            getattr(L, f).restype = ctypes.c_uint32
            getattr(L, f).argtypes = [vp]
        L.g16_circuit_device_bytes.restype = ctypes.c_uint64
        L.g16_circuit_device_bytes.argtypes = [vp]
        L.g16_kernel_timing_report.restype = ctypes.c_size_t
        L.g16_backend_fault.argtypes = [vp]
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(2048)
    lib().g16_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != G16_OK:
        raise _ERRORS.get(rc, ProveError)("g16 status %d: %s" % (rc, last_error()))


def _buf(data):
    if isinstance(data, (bytes, bytearray)):
        return ctypes.c_char_p(bytes(data)) if isinstance(data, bytes) else (ctypes.c_char * len(data)).from_buffer(data)
    # numpy arrays and other buffer objects
    mv = memoryview(data).cast("B")
    return (ctypes.c_char * mv.nbytes).from_buffer(mv) if not mv.readonly else ctypes.c_char_p(mv.tobytes())


def _nbytes(data):
    return memoryview(data).nbytes


# ---- StageTimings (crates/groth16/src/lib.rs:322-338) ----
class StageTimings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("gather_us", "ntt_us", "pointwise_us", "msm_us", "assemble_us", "verify_us")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class _Proof(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint8 * 64), ("b", ctypes.c_uint8 * 128), ("c", ctypes.c_uint8 * 64)]


class _Tuning(ctypes.Structure):
    _fields_ = [("msm_window_bits_witness", ctypes.c_int32), ("msm_window_bits_h", ctypes.c_int32),
                ("ntt_tile_log", ctypes.c_int32), ("ntt_outer_log_l", ctypes.c_int32),
                ("model_ms", ctypes.c_double), ("tuned_ms", ctypes.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class _MsmOutputs(ctypes.Structure):
    _fields_ = [("a_g1", ctypes.c_uint8 * 64), ("b_g2", ctypes.c_uint8 * 128), ("b_g1", ctypes.c_uint8 * 64),
                ("l_g1", ctypes.c_uint8 * 64), ("h_g1", ctypes.c_uint8 * 64)]


class Proof:
    """Proof{a: G1Affine, b: G2Affine, c: G1Affine} (crates/groth16/src/lib.rs:187-192), packed bytes."""

    def __init__(self, a, b, c):
        self.a, self.b, self.c = bytes(a), bytes(b), bytes(c)

    def to_bytes(self):
        return self.a + self.b + self.c

    def __eq__(self, other):
        return isinstance(other, Proof) and self.to_bytes() == other.to_bytes()

    def __repr__(self):
        return "Proof(a=%s.., b=%s.., c=%s..)" % (self.a[:4].hex(), self.b[:4].hex(), self.c[:4].hex())


def _proof_struct(proof):
    raw = proof.to_bytes() if isinstance(proof, Proof) else bytes(proof)
    if len(raw) != 256:
        raise InvalidArgumentError("a proof is 256 bytes (A 64, B 128, C 64)")
    p = _Proof()
    ctypes.memmove(ctypes.addressof(p), raw, 256)
    return p


def verify(vk, public_mont, proof):
    """verify::verify (crates/groth16/src/verify.rs:49-51) on the host.

    vk = (alpha_g1, beta_g2, gamma_g2, delta_g2, [ic points]) packed bytes;
    public_mont: the public inputs, Montgomery Fr.  Raises VerifyError,
    FormatError (unsafe key) or InvalidArgumentError (count mismatch)."""
    alpha, beta, gamma, delta, ic = vk
    icb = b"".join(ic)
    check(lib().g16_verify(bytes(alpha), bytes(beta), bytes(gamma), bytes(delta), icb, ctypes.c_size_t(len(ic)),
                           bytes(public_mont), ctypes.c_size_t(len(public_mont) // 32),
                           ctypes.byref(_proof_struct(proof))))


def pairing_check(g1_points, g2_points):
    """prod e(P_i, Q_i) == 1 over packed affine pairs."""
    if len(g1_points) != len(g2_points):
        raise InvalidArgumentError("pairing_check needs as many G1 as G2 points")
    rc = lib().g16_pairing_check(b"".join(g1_points), b"".join(g2_points), ctypes.c_size_t(len(g1_points)))
    if rc < 0:
        check(-rc)
    return rc == 1


class MsmOutputs:
    """MsmOutputs (crates/groth16/src/lib.rs:311-318): five affine points, packed."""

    FIELDS = ("a_g1", "b_g2", "b_g1", "l_g1", "h_g1")

    def __init__(self, raw):
        for f in self.FIELDS:
            setattr(self, f, bytes(getattr(raw, f)))

    def as_dict(self):
        return {f: getattr(self, f) for f in self.FIELDS}


class _ZkeyView(ctypes.Structure):
    P = ctypes.POINTER(ctypes.c_uint8)
    U = ctypes.POINTER(ctypes.c_uint32)
    _fields_ = [("n_vars", ctypes.c_uint32), ("n_public", ctypes.c_uint32), ("domain_size", ctypes.c_uint32),
                ("alpha_g1", P), ("beta_g1", P), ("beta_g2", P), ("gamma_g2", P), ("delta_g1", P), ("delta_g2", P),
                ("ic", P), ("row_ptr", U * 2), ("signal", U * 2), ("value_id", U * 2), ("nnz", ctypes.c_uint32 * 2),
                ("values", P), ("n_values", ctypes.c_uint32),
                ("a_query", P), ("b_g1_query", P), ("b_g2_query", P), ("l_query", P), ("h_query", P),
                ("h_basis", ctypes.c_uint32)]


class _KeyPlan(ctypes.Structure):
    _fields_ = [("window_tables", ctypes.c_int), ("msm_window_bits_witness", ctypes.c_int),
                ("msm_window_bits_h", ctypes.c_int), ("key_bytes", ctypes.c_uint64),
                ("workspace_bytes", ctypes.c_uint64)]


class ProvingKey:
    """A parsed snarkjs .zkey (ProvingKey, crates/formats/src/lib.rs:35-65)."""

    def __init__(self, handle):
        self._h = handle
        self._view = _ZkeyView()
        check(lib().g16_zkey_view_get(self._h, ctypes.byref(self._view)))
        self.n_vars = self._view.n_vars
        self.n_public = self._view.n_public
        self.domain_size = self._view.domain_size

    @classmethod
    def from_bytes(cls, data, check_points=True):
        """ProvingKey::from_bytes / load (check_points) / load_unchecked (not check_points)."""
        h = ctypes.c_void_p()
        check(lib().g16_zkey_parse(_buf(data), ctypes.c_size_t(_nbytes(data)), int(bool(check_points)),
                                   ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_gnark(cls, pk_dump, vk):
        """A gnark v0.14 key: the proving key's WriteDump bytes and the verifying key's
        WriteTo bytes (crates/gnark).  Proves only from A.w and B.w rows."""
        h = ctypes.c_void_p()
        check(lib().g16_gnark_key_parse(_buf(pk_dump), ctypes.c_size_t(_nbytes(pk_dump)), _buf(vk),
                                        ctypes.c_size_t(_nbytes(vk)), ctypes.byref(h)))
        return cls(h)

    @property
    def gnark(self):
        """True for gnark's bit-reversed H basis (HBasis::GnarkBitReversed)."""
        return self._view.h_basis == 1

    def query_bytes(self, name):
        """One of the five query sections as packed bytes (a_query, b_g1_query, b_g2_query,
        l_query, h_query)."""
        v = self._view
        n = {"a_query": v.n_vars * 64, "b_g1_query": v.n_vars * 64, "b_g2_query": v.n_vars * 128,
             "l_query": (v.n_vars - v.n_public - 1) * 64,
             "h_query": (v.domain_size - (1 if v.h_basis == 1 else 0)) * 64}[name]
        return ctypes.string_at(getattr(v, name), n)

    @classmethod
    def load(cls, path, check_points=True):
        with open(path, "rb") as f:
            return cls.from_bytes(f.read(), check_points)

    def plan(self, free_bytes):
        """How prepare would hold this key with free_bytes of device memory:
        {window_tables, msm_window_bits_witness, msm_window_bits_h, key_bytes,
        workspace_bytes} (host only; DeviceMemoryError when nothing fits)."""
        out = _KeyPlan()
        check(lib().g16_plan_key(ctypes.byref(self._view), ctypes.c_uint64(free_bytes), ctypes.byref(out)))
        return {n: getattr(out, n) for n, _ in out._fields_}

    def _point(self, name, size):
        return ctypes.string_at(getattr(self._view, name), size)

    @property
    def alpha_g1(self):
        return self._point("alpha_g1", 64)

    @property
    def beta_g2(self):
        return self._point("beta_g2", 128)

    @property
    def gamma_g2(self):
        return self._point("gamma_g2", 128)

    @property
    def delta_g2(self):
        return self._point("delta_g2", 128)

    @property
    def ic(self):
        raw = ctypes.string_at(self._view.ic, 64 * (self.n_public + 1))
        return [raw[64 * i:64 * i + 64] for i in range(self.n_public + 1)]

    def verifying_key(self):
        """(alpha_g1, beta_g2, gamma_g2, delta_g2, ic) packed, for verify()."""
        return self.alpha_g1, self.beta_g2, self.gamma_g2, self.delta_g2, self.ic

    def close(self):
        if self._h:
            lib().g16_zkey_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_witness(data):
    """Witness::load from .wtns bytes -> Montgomery bytes (crates/formats/src/wtns.rs:17-40)."""
    n = ctypes.c_size_t()
    check(lib().g16_wtns_parse(_buf(data), ctypes.c_size_t(_nbytes(data)), None, ctypes.c_size_t(0), ctypes.byref(n)))
    out = ctypes.create_string_buffer(32 * n.value)
    check(lib().g16_wtns_parse(_buf(data), ctypes.c_size_t(_nbytes(data)), out, n, ctypes.byref(n)))
    return out.raw


def write_witness(w_mont):
    n = _nbytes(w_mont) // 32
    ln = ctypes.c_size_t()
    check(lib().g16_wtns_write(_buf(w_mont), ctypes.c_size_t(n), None, ctypes.c_size_t(0), ctypes.byref(ln)))
    out = ctypes.create_string_buffer(ln.value)
    check(lib().g16_wtns_write(_buf(w_mont), ctypes.c_size_t(n), out, ln, ctypes.byref(ln)))
    return out.raw


class HPoly:
    """HPoly::Device (crates/groth16/src/lib.rs:207-308): H on the device, valid only on its circuit."""

    def __init__(self, handle, circuit):
        self._h = handle
        self.circuit = circuit
        self.len = circuit.domain_size

    def close(self):
        if self._h:
            lib().g16_hpoly_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaCircuit:
    """PreparedCircuit on the B200 (crates/groth16/src/lib.rs:371-455; crates/cuda/src/backend.rs CudaCircuit)."""

    def __init__(self, backend, handle, key):
        self.backend = backend
        self._h = handle
        self._key = key
        self.n_vars = lib().g16_circuit_n_vars(handle)
        self.n_public = lib().g16_circuit_n_public(handle)
        self.domain_size = lib().g16_circuit_domain_size(handle)

    def backend_name(self):
        return "cuda-b200"

    def key(self):
        return self._key

    def device_bytes(self):
        return lib().g16_circuit_device_bytes(self._h)

    def window_tables(self):
        """True when the key is held with window tables, False for a compact key."""
        return bool(lib().g16_circuit_window_tables(self._h))

    def compute_h(self, witness_mont):
        h = ctypes.c_void_p()
        check(lib().g16_compute_h(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                                  ctypes.byref(h)))
        return HPoly(h, self)

    def h_to_host(self, hpoly):
        out = ctypes.create_string_buffer(32 * hpoly.len)
        check(lib().g16_h_to_host(hpoly._h, out, ctypes.c_size_t(hpoly.len)))
        return out.raw

    def msms(self, witness_mont, hpoly):
        o = _MsmOutputs()
        check(lib().g16_msms(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32), hpoly._h,
                             ctypes.byref(o)))
        return MsmOutputs(o)

    def h_and_msms(self, witness_mont):
        o = _MsmOutputs()
        check(lib().g16_h_and_msms(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                                   ctypes.byref(o)))
        return MsmOutputs(o)

    def prove_with_blinders(self, witness_mont, r_mont, s_mont):
        """prove_with_blinders (crates/groth16/src/prove.rs:175-184); r, s: 32-byte Montgomery Fr."""
        p = _Proof()
        check(lib().g16_prove_with_blinders(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                                            bytes(r_mont), bytes(s_mont), ctypes.byref(p)))
        return Proof(p.a, p.b, p.c)

    def warm(self, count):
        """Ready up to `count` workspaces (g16_circuit_warm): that many concurrent
        proofs then allocate nothing and replay CUDA graphs."""
        check(lib().g16_circuit_warm(self._h, ctypes.c_uint32(count)))

    def prove_with_blinders_device(self, d_witness, n, r_mont, s_mont):
        p = _Proof()
        check(lib().g16_prove_with_blinders_device(self._h, ctypes.c_void_p(d_witness), ctypes.c_size_t(n),
                                                   bytes(r_mont), bytes(s_mont), ctypes.byref(p)))
        return Proof(p.a, p.b, p.c)

    def set_serial(self, serial=True):
        """Run every stage on one stream (profiling); results are identical."""
        check(lib().g16_circuit_set_serial(self._h, int(bool(serial))))

    def readback_bytes(self):
        lib().g16_circuit_readback_bytes.restype = ctypes.c_uint64
        return lib().g16_circuit_readback_bytes(self._h)

    def stage_timings(self):
        t = StageTimings()
        check(lib().g16_stage_timings_get(self._h, ctypes.byref(t)))
        return t.as_dict()

    def h_and_msms_from_rows(self, witness_mont, a_rows, b_rows):
        """PreparedCircuit::h_and_msms_from_rows: stage 0 handed over as A.w and B.w rows."""
        if _nbytes(a_rows) != _nbytes(b_rows):
            raise BackendError("A.w and B.w must have the same number of rows")
        o = _MsmOutputs()
        check(lib().g16_h_and_msms_from_rows(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                                             _buf(a_rows), _buf(b_rows), ctypes.c_size_t(_nbytes(a_rows) // 32),
                                             ctypes.byref(o)))
        return MsmOutputs(o)

    def prove_with_blinders_from_rows(self, witness_mont, a_rows, b_rows, r_mont, s_mont):
        if _nbytes(a_rows) != _nbytes(b_rows):
            raise BackendError("A.w and B.w must have the same number of rows")
        p = _Proof()
        check(lib().g16_prove_with_blinders_from_rows(self._h, _buf(witness_mont),
                                                      ctypes.c_size_t(_nbytes(witness_mont) // 32), _buf(a_rows),
                                                      _buf(b_rows), ctypes.c_size_t(_nbytes(a_rows) // 32),
                                                      bytes(r_mont), bytes(s_mont), ctypes.byref(p)))
        return Proof(p.a, p.b, p.c)

    def prove(self, witness_mont):
        """prove::prove (crates/groth16/src/prove.rs:34-92): fresh r, s, then the proof is checked."""
        p = _Proof()
        check(lib().g16_prove(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                              ctypes.byref(p)))
        return Proof(p.a, p.b, p.c)

    def verify(self, public_mont, proof):
        """verify::verify against this circuit's key; raises VerifyError when the proof fails."""
        check(lib().g16_circuit_verify(self._h, bytes(public_mont), ctypes.c_size_t(len(public_mont) // 32),
                                       ctypes.byref(_proof_struct(proof))))

    def tuning(self):
        """MSM window bits and NTT tiling in use (cost model, autotuner or set_tuning)."""
        t = _Tuning()
        check(lib().g16_tuning_get(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, msm_window_bits_witness, msm_window_bits_h, ntt_tile_log, ntt_outer_log_l):
        t = _Tuning(msm_window_bits_witness, msm_window_bits_h, ntt_tile_log, ntt_outer_log_l, 0.0, 0.0)
        check(lib().g16_tuning_set(self._h, ctypes.byref(t)))

    def autotune(self, witness_mont, concurrency=1):
        """Time window sizes and NTT tilings with this witness on the device; keep the fastest.

        concurrency 1: one proof's latency; 2..8: device time per proof with
        that many proofs in flight together (batched / served proving)."""
        t = _Tuning()
        check(lib().g16_autotune(self._h, _buf(witness_mont), ctypes.c_size_t(_nbytes(witness_mont) // 32),
                                 int(concurrency), ctypes.byref(t)))
        return t.as_dict()

    def close(self):
        if self._h:
            lib().g16_circuit_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaBackend:
    """Backend (crates/groth16/src/lib.rs:371-380) over one B200: name() and prepare()."""

    def __init__(self, ordinal=0, vram_limit=0, constant_work=False):
        self.ordinal = int(ordinal)
        h = ctypes.c_void_p()
        check(lib().g16_backend_open(int(ordinal), ctypes.c_uint64(vram_limit), ctypes.byref(h)))
        self._h = h
        if constant_work:
            self.set_constant_work(True)

    @classmethod
    def constant_work(cls, ordinal=0, vram_limit=0):
        """CudaBackend::constant_work (crates/cuda/src/backend.rs:100-118)."""
        return cls(ordinal, vram_limit, constant_work=True)

    def set_constant_work(self, on=True):
        """MSM cost follows the key, not the witness (results unchanged)."""
        check(lib().g16_backend_set_constant_work(self._h, int(bool(on))))

    def name(self):
        return lib().g16_backend_name(self._h).decode()

    def batch_stats(self):
        """Counters of the batched-proving engines: submissions, new layouts,
        graph replays, device bytes grown, engines built."""
        st = _BatchStats()
        check(lib().g16_batch_stats_get(self._h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in st._fields_}

    def batch_reserve(self, circuits):
        """Size every batched-proving engine for a batch of these circuits (repeats
        allowed) without proving it: a later prove_batch of that mix allocates no
        device memory (g16_batch_reserve)."""
        n = len(circuits)
        arr = (ctypes.c_void_p * max(n, 1))(*[c._h for c in circuits])
        check(lib().g16_batch_reserve(self._h, ctypes.c_size_t(n), arr))

    def fault(self):
        """The sticky cudaError_t value that put this backend out of use, or 0."""
        return lib().g16_backend_fault(self._h)

    def inject_fault(self, cuda_error):
        """The next device entry point on this backend fails as if the driver had
        returned cuda_error; no device work happens (a host-side test hook)."""
        check(lib().g16_backend_inject_fault(self._h, int(cuda_error)))

    def vram_used(self):
        return lib().g16_backend_vram_used(self._h)

    def prepare(self, pk):
        c = ctypes.c_void_p()
        check(lib().g16_prepare(self._h, ctypes.byref(pk._view), ctypes.byref(c)))
        return CudaCircuit(self, c, pk)

    def prove_batch(self, jobs, done_ms=None):
        """Prove [(circuit, witness_mont, r_mont, s_mont), ...] in one submission.

        done_ms: an optional list that receives, per job, the milliseconds from the
        submission until that proof was complete."""
        n = len(jobs)
        circ = (ctypes.c_void_p * n)(*[j[0]._h for j in jobs])
        bufs = [bytes(j[1]) for j in jobs]
        wits = (ctypes.c_char_p * n)(*bufs)
        lens = (ctypes.c_size_t * n)(*[len(b) // 32 for b in bufs])
        r = b"".join(bytes(j[2]) for j in jobs)
        s = b"".join(bytes(j[3]) for j in jobs)
        out = (_Proof * n)()
        done = (ctypes.c_double * max(n, 1))()
        check(lib().g16_prove_batch_timed(self._h, ctypes.c_size_t(n), circ, wits, lens, r, s, out, done))
        if done_ms is not None:
            done_ms[:] = list(done)[:n]
        return [Proof(p.a, p.b, p.c) for p in out]

    # device memory helpers
    def alloc(self, nbytes):
        d = ctypes.c_void_p()
        check(lib().g16_device_alloc(self._h, ctypes.c_size_t(nbytes), ctypes.byref(d)))
        return d.value

    def free(self, d):
        check(lib().g16_device_free(self._h, ctypes.c_void_p(d)))

    def upload(self, d, data):
        check(lib().g16_device_upload(self._h, ctypes.c_void_p(d), _buf(data), ctypes.c_size_t(_nbytes(data))))

    def sync(self):
        check(lib().g16_device_sync(self._h))

    def close(self):
        if self._h:
            lib().g16_backend_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("submitted", "completed", "prepared", "evicted", "resident_keys", "resident_bytes", "queued",
                 "batches", "batched", "alone")]


class _BatchStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submissions", "layouts", "replays", "grown_bytes", "engines")]


class ProofServer:
    """Served proving with continuous batching over a set of registered keys."""

    def __init__(self, backend, key_budget_bytes=0, lanes=4, max_batch=64):
        """lanes: concurrent batches; max_batch: requests per batch (1 = plain one-at-a-time)."""
        h = ctypes.c_void_p()
        check(lib().g16_server_new(backend._h, ctypes.c_uint64(key_budget_bytes), int(lanes), ctypes.byref(h)))
        self._h = h
        self.backend = backend
        check(lib().g16_server_set_max_batch(h, ctypes.c_size_t(max_batch)))

    def register_key(self, key_id, zkey_bytes):
        check(lib().g16_server_register_key(self._h, ctypes.c_uint32(key_id), bytes(zkey_bytes),
                                            ctypes.c_size_t(len(zkey_bytes))))

    def submit(self, key_id, witness_mont, r_mont, s_mont):
        t = ctypes.c_uint64()
        check(lib().g16_server_submit(self._h, ctypes.c_uint32(key_id), _buf(witness_mont),
                                      ctypes.c_size_t(_nbytes(witness_mont) // 32), bytes(r_mont), bytes(s_mont),
                                      ctypes.byref(t)))
        return t.value

    def wait(self, ticket):
        """(Proof, queue_ms, latency_ms)."""
        p = _Proof()
        q, lat = ctypes.c_double(), ctypes.c_double()
        check(lib().g16_server_wait(self._h, ctypes.c_uint64(ticket), ctypes.byref(p), ctypes.byref(q),
                                    ctypes.byref(lat)))
        return Proof(p.a, p.b, p.c), q.value, lat.value

    def stats(self):
        st = _ServerStats()
        check(lib().g16_server_stats_get(self._h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in st._fields_}

    def close(self):
        if self._h:
            lib().g16_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CudaMsm:
    """MsmBackend (crates/msm/src/lib.rs:52-82) on the B200."""

    def __init__(self, backend):
        self.backend = backend

    def name(self):
        return "cuda-b200"

    def _run(self, fn, size, bases, scalars, form):
        n = _nbytes(scalars) // 32
        if _nbytes(bases) != n * size:
            raise BackendError("MSM length mismatch: %d bases but %d scalars" % (_nbytes(bases) // size, n))
        out = ctypes.create_string_buffer(size)
        check(fn(self.backend._h, _buf(bases), _buf(scalars), ctypes.c_size_t(n), int(form), out))
        return out.raw

    def msm_g1(self, bases, scalars, form=SCALARS_STANDARD):
        return self._run(lib().g16_msm_g1, 64, bases, scalars, form)

    def msm_g2(self, bases, scalars, form=SCALARS_STANDARD):
        return self._run(lib().g16_msm_g2, 128, bases, scalars, form)

    try_msm_g1 = msm_g1
    try_msm_g2 = msm_g2

    def msm_g1_device(self, d_bases, d_scalars, n, form=SCALARS_STANDARD):
        out = ctypes.create_string_buffer(64)
        check(lib().g16_msm_g1_device(self.backend._h, ctypes.c_void_p(d_bases), ctypes.c_void_p(d_scalars),
                                      ctypes.c_size_t(n), int(form), out))
        return out.raw

    def msm_g1_device_noalloc(self, d_bases, d_scalars, n, form=SCALARS_STANDARD):
        """G1 MSM that allocates nothing (fixed library scratch, at most 16384 points)."""
        out = ctypes.create_string_buffer(64)
        check(lib().g16_msm_g1_device_noalloc(ctypes.c_int(self.backend.ordinal), ctypes.c_void_p(d_bases),
                                              ctypes.c_void_p(d_scalars), ctypes.c_size_t(n), int(form), out))
        return out.raw

    def msm_g2_device(self, d_bases, d_scalars, n, form=SCALARS_STANDARD):
        out = ctypes.create_string_buffer(128)
        check(lib().g16_msm_g2_device(self.backend._h, ctypes.c_void_p(d_bases), ctypes.c_void_p(d_scalars),
                                      ctypes.c_size_t(n), int(form), out))
        return out.raw


class CudaNtt:
    """The CpuNtt API (crates/ntt/src/lib.rs:415-584) on the B200; data is Montgomery bytes, in place semantics."""

    def __init__(self, backend):
        self.backend = backend

    def _run(self, mode, data, shift_mont=None):
        n = _nbytes(data) // 32
        log_n = n.bit_length() - 1
        if n < 2 or (1 << log_n) != n:
            raise InvalidArgumentError("NTT length %d is not a power of two >= 2" % n)
        buf = ctypes.create_string_buffer(bytes(data), _nbytes(data))
        sh = None if shift_mont is None else bytes(shift_mont)
        check(lib().g16_ntt(self.backend._h, int(mode), ctypes.c_uint32(log_n), buf, sh))
        return buf.raw

    def ntt(self, data, inverse=False):
        return self._run(NTT_INVERSE if inverse else NTT_FORWARD, data)

    def intt_coset_ntt(self, data):
        return self._run(NTT_INTT_COSET_NTT, data)

    def coset_ntt(self, data, shift_mont=None, inverse=False):
        return self._run(NTT_COSET_INVERSE if inverse else NTT_COSET_FORWARD, data, shift_mont)

    def ntt_device(self, mode, log_n, d_data, shift_mont=None):
        sh = None if shift_mont is None else bytes(shift_mont)
        check(lib().g16_ntt_device(self.backend._h, int(mode), ctypes.c_uint32(log_n), ctypes.c_void_p(d_data), sh))


class SynthCircuit:
    """A seeded synthetic R1CS with its witness generator and toxic-waste .zkey writer."""

    def __init__(self, seed, n_constraints, n_inputs=256, n_public=16):
        h = ctypes.c_void_p()
        check(lib().g16_synth_new(ctypes.c_uint64(seed), ctypes.c_uint32(n_constraints), ctypes.c_uint32(n_inputs),
                                  ctypes.c_uint32(n_public), ctypes.byref(h)))
        self._h = h
        self.n_public = n_public
        self.n_vars = lib().g16_synth_n_vars(h)
        self.domain_size = lib().g16_synth_domain_size(h)

    def witness(self, witness_seed):
        out = ctypes.create_string_buffer(32 * self.n_vars)
        check(lib().g16_synth_witness(self._h, ctypes.c_uint64(witness_seed), out))
        return out.raw

    def zkey(self, toxic_seed, threads=0, device=None):
        """The .zkey bytes from seeded toxic waste; device=ordinal computes the point
        sections on that GPU (the same bytes), otherwise host threads do."""
        n = ctypes.c_size_t()
        if device is None:
            fn = lambda buf, cap: lib().g16_synth_zkey(self._h, ctypes.c_uint64(toxic_seed), int(threads), buf, cap,
                                                       ctypes.byref(n))
        else:
            fn = lambda buf, cap: lib().g16_synth_zkey_device(self._h, ctypes.c_uint64(toxic_seed), int(device), buf,
                                                              cap, ctypes.byref(n))
        check(fn(None, ctypes.c_size_t(0)))
        out = ctypes.create_string_buffer(n.value)
        check(fn(out, n))
        return out.raw

    def r1cs(self):
        n = ctypes.c_size_t()
        check(lib().g16_synth_r1cs(self._h, None, ctypes.c_size_t(0), ctypes.byref(n)))
        out = ctypes.create_string_buffer(n.value)
        check(lib().g16_synth_r1cs(self._h, out, n, ctypes.byref(n)))
        return out.raw

    def close(self):
        if self._h:
            lib().g16_synth_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synth_points(group, seed, n, threads=0):
    """n affine points k_i G, k_i uniform (group 1 = G1, 2 = G2), packed bytes."""
    out = ctypes.create_string_buffer((64 if group == 1 else 128) * n)
    check(lib().g16_synth_points(int(group), ctypes.c_uint64(seed), ctypes.c_size_t(n), int(threads), out))
    return out.raw


def synth_scalars(seed, n, dist=0):
    """n standard-form scalars; dist 0 uniform, dist 1 = 70% in {0, 1}."""
    out = ctypes.create_string_buffer(32 * n)
    check(lib().g16_synth_scalars(ctypes.c_uint64(seed), ctypes.c_size_t(n), int(dist), out))
    return out.raw


def kernel_timing(enable=True):
    lib().g16_kernel_timing_enable(int(bool(enable)))


def kernel_timing_reset():
    lib().g16_kernel_timing_reset()


def _timing_lines():
    buf = ctypes.create_string_buffer(1 << 16)
    lib().g16_kernel_timing_report(buf, 1 << 16)
    return [line.split() for line in buf.value.decode().splitlines()]


def kernel_timing_report():
    """{kernel class: (total ms, launches, work units)} from CUDA events on the launching stream.

    Work units are the mixed additions performed, for the MSM accumulate kernels,
    and the Fr products, for the NTT passes."""
    return {f[0]: (float(f[1]), int(f[2]), float(f[3])) for f in _timing_lines()}


def kernel_timing_bytes():
    """{kernel class: algorithmic HBM bytes} over the same launches (NTT passes, MSM sort)."""
    return {f[0]: float(f[4]) for f in _timing_lines() if float(f[4]) > 0}


def launch_count():
    """Kernels this library has launched since it was loaded."""
    lib().g16_launch_count.restype = ctypes.c_uint64
    return lib().g16_launch_count()


def gnark_witness(data):
    """A gnark witness dump (W, A.w, B.w; crates/gnark/src/witness.rs) as three byte
    strings of Montgomery Fr."""
    n_w, n_rows = ctypes.c_size_t(), ctypes.c_size_t()
    check(lib().g16_gnark_witness_parse(_buf(data), ctypes.c_size_t(_nbytes(data)), None, ctypes.c_size_t(0), None,
                                        None, ctypes.c_size_t(0), ctypes.byref(n_w), ctypes.byref(n_rows)))
    w = ctypes.create_string_buffer(32 * n_w.value)
    aw = ctypes.create_string_buffer(32 * n_rows.value)
    bw = ctypes.create_string_buffer(32 * n_rows.value)
    check(lib().g16_gnark_witness_parse(_buf(data), ctypes.c_size_t(_nbytes(data)), w, n_w, aw, bw, n_rows, None,
                                        None))
    return w.raw, aw.raw, bw.raw


FAULT_DEVICE, FAULT_STICKY = 1, 2


def cuda_error_class(cuda_error):
    """FAULT_DEVICE / FAULT_STICKY classes of a cudaError_t value (is_device_fault and
    is_sticky, crates/cuda/src/context.rs:134-215).  Needs no device."""
    return lib().g16_cuda_error_class(int(cuda_error))


def device_alloc_count():
    """Device allocations (cudaMalloc calls) this library has made since it was loaded."""
    lib().g16_device_alloc_count.restype = ctypes.c_uint64
    return lib().g16_device_alloc_count()


def imad_peak(backend):
    """Measured 32-bit mad.lo/mad.hi issue rate of the device (per second)."""
    v = ctypes.c_double()
    check(lib().g16_imad_peak(backend._h, ctypes.byref(v)))
    return v.value


def fr_to_mont_bytes(x):
    return ((int(x) << 256) % R_MOD).to_bytes(32, "little")


def fr_from_mont_bytes(b):
    return int.from_bytes(bytes(b), "little") * pow(1 << 256, -1, R_MOD) % R_MOD
