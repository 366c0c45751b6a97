"""CPU ORACLE -- test infrastructure only.

ctypes bindings for ``oracle/liboracle.so``, the plain-C restatement of the
reference CPU prover (zemse/snarkrs ``crates/groth16/src/cpu.rs``,
``crates/ntt``, ``crates/msm``, ``crates/groth16/src/verify.rs``).  Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg load
this module; the product never does.

Byte conventions: field elements are 32 little-endian bytes (Montgomery form
unless a name says ``std``); G1 points are 64 bytes (x||y), G2 points 128
bytes (x.c0||x.c1||y.c0||y.c1), infinity all-zero; a proof is A||B||C
(256 bytes).
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()   # make rebuilds only when a source is newer than the library
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_init()
        _lib.oracle_zkey_load.restype = ctypes.c_void_p
        _lib.oracle_zkey_load.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
        _lib.oracle_zkey_free.argtypes = [ctypes.c_void_p]
        _lib.oracle_zkey_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        for name in ("oracle_compute_h", "oracle_msms", "oracle_prove", "oracle_verify_zkey"):
            getattr(_lib, name).argtypes = None
        _lib.oracle_msm_g1.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
        _lib.oracle_msm_g2.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
    return _lib


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return lib().oracle_max_threads()


# ---- integer <-> bytes helpers ----
def to_bytes(x):
    return int(x).to_bytes(32, "little")


def from_bytes(b):
    return int.from_bytes(bytes(b), "little")


def to_mont(x, mod=R_MOD):
    return (int(x) << 256) % mod


def from_mont(x, mod=R_MOD):
    return (int(x) * pow(1 << 256, -1, mod)) % mod


# ---- field ----
def field_consts(which):
    p = ctypes.create_string_buffer(32)
    n0 = ctypes.c_uint64()
    one = ctypes.create_string_buffer(32)
    r2 = ctypes.create_string_buffer(32)
    lib().oracle_field_consts(which, p, ctypes.byref(n0), one, r2)
    return from_bytes(p.raw), n0.value, from_bytes(one.raw), from_bytes(r2.raw)


def fp_op(op, which, a, b=None):
    out = ctypes.create_string_buffer(32)
    fn = getattr(lib(), "oracle_fp_" + op)
    if b is None:
        fn(which, to_bytes(a), out)
    else:
        fn(which, to_bytes(a), to_bytes(b), out)
    return from_bytes(out.raw)


def fq2_mul(a, b):
    out = ctypes.create_string_buffer(64)
    lib().oracle_fq2_mul(to_bytes(a[0]) + to_bytes(a[1]), to_bytes(b[0]) + to_bytes(b[1]), out)
    return (from_bytes(out.raw[:32]), from_bytes(out.raw[32:]))


def hard_exponent():
    arr = (ctypes.c_uint32 * 40)()
    lib().oracle_hard_exponent(arr)
    return sum(int(v) << (32 * i) for i, v in enumerate(arr))


def domain_root(log_n):
    out = ctypes.create_string_buffer(32)
    if lib().oracle_domain_root(log_n, out) != 0:
        raise ValueError("no root of that order")
    return from_bytes(out.raw)   # Montgomery


# ---- NTT (data: bytes of n Montgomery elements) ----
NTT_FORWARD, NTT_INVERSE, NTT_INTT_COSET_NTT, NTT_COSET_FORWARD, NTT_COSET_INVERSE = range(5)


def ntt(log_n, mode, data, shift_mont=None):
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    sh = None if shift_mont is None else ctypes.create_string_buffer(to_bytes(shift_mont), 32)
    if lib().oracle_ntt(log_n, mode, buf, sh) != 0:
        raise ValueError("bad NTT request")
    return buf.raw


# ---- curve ----
def g1_generator():
    out = ctypes.create_string_buffer(64)
    lib().oracle_g1_generator(out)
    return out.raw


def g2_generator():
    out = ctypes.create_string_buffer(128)
    lib().oracle_g2_generator(out)
    return out.raw


def g1_mul(p, k):
    out = ctypes.create_string_buffer(64)
    if lib().oracle_g1_mul(bytes(p), to_bytes(k % R_MOD), out) != 0:
        raise ValueError("bad point")
    return out.raw


def g2_mul(p, k):
    out = ctypes.create_string_buffer(128)
    if lib().oracle_g2_mul(bytes(p), to_bytes(k % R_MOD), out) != 0:
        raise ValueError("bad point")
    return out.raw


def g1_add(p, q):
    out = ctypes.create_string_buffer(64)
    lib().oracle_g1_add(bytes(p), bytes(q), out)
    return out.raw


def g2_add(p, q):
    out = ctypes.create_string_buffer(128)
    lib().oracle_g2_add(bytes(p), bytes(q), out)
    return out.raw


def g1_on_curve(p):
    return bool(lib().oracle_g1_on_curve(bytes(p)))


def g2_on_curve(p):
    return bool(lib().oracle_g2_on_curve(bytes(p)))


def g2_in_subgroup(p):
    return bool(lib().oracle_g2_in_subgroup(bytes(p)))


def pairing_check(g1s, g2s):
    n = len(g1s)
    r = lib().oracle_pairing_check(b"".join(g1s), b"".join(g2s), n)
    if r < 0:
        raise ValueError("bad point")
    return bool(r)


# ---- MSM ----
def msm_g1(bases, scalars_std):
    """bases: bytes (64 per point); scalars_std: bytes (32 per scalar, standard form)."""
    n = len(bases) // 64
    out = ctypes.create_string_buffer(64)
    if lib().oracle_msm_g1(bytes(bases), bytes(scalars_std), n, out) != 0:
        raise ValueError("bad base")
    return out.raw


def msm_g2(bases, scalars_std):
    n = len(bases) // 128
    out = ctypes.create_string_buffer(128)
    if lib().oracle_msm_g2(bytes(bases), bytes(scalars_std), n, out) != 0:
        raise ValueError("bad base")
    return out.raw


# ---- zkey / prover ----
class Zkey:
    """A zkey parsed by the oracle's own reader (independent of the product's)."""

    def __init__(self, data, _handle=None):
        if _handle is None:
            err = ctypes.create_string_buffer(256)
            _handle = lib().oracle_zkey_load(bytes(data), len(data), err, 256)
            if not _handle:
                raise ValueError(err.value.decode())
        self._h = _handle
        info = (ctypes.c_uint32 * 3)()
        lib().oracle_zkey_info(ctypes.c_void_p(self._h), info)
        self.n_vars, self.n_public, self.domain_size = info[0], info[1], info[2]
        self.gnark = bool(lib().oracle_zkey_h_basis(ctypes.c_void_p(self._h)))

    @classmethod
    def from_gnark(cls, pk_dump, vk):
        """A gnark v0.14 proving-key dump and verifying key (the bit-reversed H basis)."""
        err = ctypes.create_string_buffer(256)
        L = lib()
        L.oracle_gnark_load.restype = ctypes.c_void_p
        h = L.oracle_gnark_load(bytes(pk_dump), ctypes.c_size_t(len(pk_dump)), bytes(vk), ctypes.c_size_t(len(vk)),
                                err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(None, _handle=h)

    def query(self, which):
        """A query packed: 'a', 'b1', 'b2', 'l' or 'h'."""
        i = ["a", "b1", "b2", "l", "h"].index(which)
        L = lib()
        L.oracle_zkey_query.restype = ctypes.c_size_t
        n = L.oracle_zkey_query(ctypes.c_void_p(self._h), i, None)
        out = ctypes.create_string_buffer(n * (128 if which == "b2" else 64))
        L.oracle_zkey_query(ctypes.c_void_p(self._h), i, out)
        return out.raw

    def vk_bytes(self):
        """alpha_g1 | beta_g2 | gamma_g2 | delta_g2 | ic, packed."""
        L = lib()
        L.oracle_zkey_vk.restype = ctypes.c_size_t
        n = L.oracle_zkey_vk(ctypes.c_void_p(self._h), None)
        out = ctypes.create_string_buffer(n)
        L.oracle_zkey_vk(ctypes.c_void_p(self._h), out)
        return out.raw

    def prove_rows(self, witness_mont, a_rows, b_rows, r_mont, s_mont):
        """Stages 1-11 from A.w and B.w rows (either H basis)."""
        out = ctypes.create_string_buffer(256)
        rc = lib().oracle_prove_rows(ctypes.c_void_p(self._h), bytes(witness_mont),
                                     ctypes.c_size_t(len(witness_mont) // 32), bytes(a_rows), bytes(b_rows),
                                     ctypes.c_size_t(len(a_rows) // 32), to_bytes(r_mont), to_bytes(s_mont), out)
        if rc != 0:
            raise ValueError("prove_rows failed")
        return out.raw

    def close(self):
        if self._h:
            lib().oracle_zkey_free(ctypes.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute_h(self, witness_mont):
        out = ctypes.create_string_buffer(32 * self.domain_size)
        rc = lib().oracle_compute_h(ctypes.c_void_p(self._h), bytes(witness_mont),
                                    ctypes.c_size_t(len(witness_mont) // 32), out)
        if rc != 0:
            raise ValueError("compute_h failed")
        return out.raw

    def gather(self, witness_mont):
        """Stage 0: (A.w, B.w), domain_size rows each, Montgomery bytes."""
        a = ctypes.create_string_buffer(32 * self.domain_size)
        b = ctypes.create_string_buffer(32 * self.domain_size)
        rc = lib().oracle_gather(ctypes.c_void_p(self._h), bytes(witness_mont),
                                 ctypes.c_size_t(len(witness_mont) // 32), a, b)
        if rc != 0:
            raise ValueError("gather failed")
        return a.raw, b.raw

    def compute_h_from_rows(self, a_rows, b_rows):
        out = ctypes.create_string_buffer(32 * self.domain_size)
        rc = lib().oracle_compute_h_from_rows(ctypes.c_void_p(self._h), bytes(a_rows), bytes(b_rows),
                                              ctypes.c_size_t(len(a_rows) // 32), out)
        if rc != 0:
            raise ValueError("compute_h_from_rows failed")
        return out.raw

    def msms(self, witness_mont, h_mont):
        out = ctypes.create_string_buffer(384)
        rc = lib().oracle_msms(ctypes.c_void_p(self._h), bytes(witness_mont),
                               ctypes.c_size_t(len(witness_mont) // 32), bytes(h_mont), out)
        if rc != 0:
            raise ValueError("msms failed")
        b = out.raw
        return {"a_g1": b[:64], "b_g2": b[64:192], "b_g1": b[192:256], "l_g1": b[256:320], "h_g1": b[320:384]}

    def prove(self, witness_mont, r_mont, s_mont):
        out = ctypes.create_string_buffer(256)
        rc = lib().oracle_prove(ctypes.c_void_p(self._h), bytes(witness_mont),
                                ctypes.c_size_t(len(witness_mont) // 32), to_bytes(r_mont), to_bytes(s_mont), out)
        if rc != 0:
            raise ValueError("prove failed")
        return out.raw

    def verify(self, public_mont, proof):
        rc = lib().oracle_verify_zkey(ctypes.c_void_p(self._h), bytes(public_mont),
                                      ctypes.c_size_t(len(public_mont) // 32), bytes(proof))
        if rc < 0:
            raise ValueError("wrong public input count")
        return bool(rc)


def gnark_witness(data):
    """A gnark witness dump (marker, then W, A.w and B.w as u64 LE count + Montgomery Fr):
    (w, a_rows, b_rows) as Montgomery bytes."""
    if len(data) < 8 or data[:8] != (0xdeadbeef).to_bytes(8, "little"):
        raise ValueError("not a gnark dump")
    off, out = 8, []
    for _ in range(3):
        n = int.from_bytes(data[off:off + 8], "little")
        off += 8
        if off + 32 * n > len(data):
            raise ValueError("truncated witness dump")
        out.append(bytes(data[off:off + 32 * n]))
        off += 32 * n
    if off != len(data):
        raise ValueError("trailing bytes")
    return tuple(out)


def verify_vk(alpha, beta, gamma, delta, ic, public_mont, proof):
    vk = bytes(alpha) + bytes(beta) + bytes(gamma) + bytes(delta) + b"".join(ic)
    rc = lib().oracle_verify_vk(vk, ctypes.c_size_t(len(ic)), bytes(public_mont), bytes(proof))
    if rc < 0:
        raise ValueError("bad verifying key")
    return bool(rc)


# ---- the timed CPU baseline (port_*.c) ----
def _port_lib():
    L = lib()
    if not getattr(L, "_port_bound", False):
        L.oracle_port_prepare.restype = ctypes.c_void_p
        L.oracle_port_prepare.argtypes = [ctypes.c_void_p]
        L.oracle_port_free.argtypes = [ctypes.c_void_p]
        L.oracle_port_prove.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                        ctypes.c_char_p, ctypes.c_char_p]
        L.oracle_port_msm_g1.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
        L.oracle_port_msm_g2.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p]
        L.oracle_port_intt_coset_ntt.argtypes = [ctypes.c_int, ctypes.c_char_p]
        L.oracle_synth_new.restype = ctypes.c_void_p
        L.oracle_synth_new.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_synth_free.argtypes = [ctypes.c_void_p]
        L.oracle_synth_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_synth_witness.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p]
        L.oracle_synth_zkey.restype = ctypes.POINTER(ctypes.c_uint8)
        L.oracle_synth_zkey.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_synth_buffer_free.argtypes = [ctypes.POINTER(ctypes.c_uint8)]
        L._port_bound = True
    return L


class PortProver:
    """The reference CPU prover's algorithms restated for speed (batch-affine MSM fill,
    the five MSMs concurrently, 2^11-blocked intt_coset_ntt): the timed CPU baseline.
    Its proofs equal the oracle's."""

    def __init__(self, zkey):
        self.zkey = zkey
        self._h = _port_lib().oracle_port_prepare(ctypes.c_void_p(zkey._h))
        if not self._h:
            raise ValueError("port prepare failed")

    def prove(self, witness_mont, r_mont, s_mont):
        """r_mont, s_mont: 32-byte Montgomery Fr."""
        out = ctypes.create_string_buffer(256)
        rc = _port_lib().oracle_port_prove(ctypes.c_void_p(self._h), bytes(witness_mont),
                                           ctypes.c_size_t(len(witness_mont) // 32), bytes(r_mont), bytes(s_mont),
                                           out)
        if rc != 0:
            raise ValueError("port prove failed")
        return out.raw

    def close(self):
        if self._h:
            _port_lib().oracle_port_free(ctypes.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def port_msm_g1(bases, scalars_std):
    out = ctypes.create_string_buffer(64)
    if _port_lib().oracle_port_msm_g1(bytes(bases), bytes(scalars_std), len(bases) // 64, out) != 0:
        raise ValueError("bad base")
    return out.raw


def port_msm_g2(bases, scalars_std):
    out = ctypes.create_string_buffer(128)
    if _port_lib().oracle_port_msm_g2(bytes(bases), bytes(scalars_std), len(bases) // 128, out) != 0:
        raise ValueError("bad base")
    return out.raw


def port_intt_coset_ntt(log_n, data):
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    if _port_lib().oracle_port_intt_coset_ntt(log_n, buf) != 0:
        raise ValueError("bad size")
    return buf.raw


class Synth:
    """The synthetic workload generator restated on the oracle's side (synth.c): the
    same seeds give the same circuit, witnesses and .zkey bytes as the product's."""

    def __init__(self, seed, n_constraints, n_inputs=256, n_public=16):
        L = _port_lib()
        self._h = L.oracle_synth_new(seed, n_constraints, n_inputs, n_public)
        if not self._h:
            raise ValueError("bad synthetic circuit shape")
        info = (ctypes.c_uint32 * 2)()
        L.oracle_synth_info(ctypes.c_void_p(self._h), info)
        self.n_vars, self.domain_size, self.n_public = info[0], info[1], n_public

    def witness(self, witness_seed):
        out = ctypes.create_string_buffer(32 * self.n_vars)
        _port_lib().oracle_synth_witness(ctypes.c_void_p(self._h), witness_seed, out)
        return out.raw

    def zkey(self, toxic_seed):
        L = _port_lib()
        n = ctypes.c_size_t()
        p = L.oracle_synth_zkey(ctypes.c_void_p(self._h), toxic_seed, ctypes.byref(n))
        try:
            return ctypes.string_at(p, n.value)
        finally:
            L.oracle_synth_buffer_free(p)

    def close(self):
        if self._h:
            _port_lib().oracle_synth_free(ctypes.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
