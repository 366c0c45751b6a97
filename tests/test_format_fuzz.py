"""The host readers behind the C ABI never crash on malformed input: g16_zkey_parse,
g16_gnark_key_parse, g16_gnark_witness_parse and g16_wtns_parse are fed a valid
file with random truncations, byte flips, and rewritten section sizes, ids and
field widths, and each call must return a status (a parsed key is viewed and
freed).  The calls run in a child process, so a crash fails this test instead of
ending the test run.  No GPU is involved."""
import gzip
import json
import os
import subprocess
import sys

import pytest

import snarkrs_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

FUZZ = r"""
import ctypes, random, struct, sys
sys.path.insert(0, sys.argv[1])
import snarkrs_b200 as S
L = S.lib()
L.g16_zkey_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
L.g16_gnark_key_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_void_p)]
L.g16_zkey_free.argtypes = [ctypes.c_void_p]
L.g16_zkey_view_get.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
L.g16_wtns_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                             ctypes.POINTER(ctypes.c_size_t)]
L.g16_gnark_witness_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
zk, pk, vk, wtns, gw = (open(p, "rb").read() for p in sys.argv[2:7])
rng = random.Random(int(sys.argv[7]))
view = ctypes.create_string_buffer(4096)

def sections(b, start):
    # (offset of the section header, id, size) for a zkey/wtns-style section table
    out, off = [], start
    while off + 12 <= len(b):
        sid, size = struct.unpack_from("<IQ", b, off)
        out.append((off, sid, size))
        off += 12 + size
    return out

def mutate(b, start):
    b = bytearray(b)
    kind = rng.randrange(5)
    if kind == 0 and len(b) > 1:
        return bytes(b[:rng.randrange(len(b))])
    if kind == 1:
        for _ in range(rng.randrange(1, 9)):
            i = rng.randrange(len(b))
            b[i] ^= 1 << rng.randrange(8)
        return bytes(b)
    secs = sections(bytes(b), start) if start is not None else []
    if kind in (2, 3) and secs:
        off, sid, size = rng.choice(secs)
        if kind == 2:
            struct.pack_into("<Q", b, off + 4, rng.choice([0, 1, 7, size - 1, size + 1, len(b), 1 << 40, (1 << 64) - 1]))
        else:
            struct.pack_into("<I", b, off, rng.choice([0, 1, 2, 3, 4, 9, 10, 11, 0xFFFFFFFF]))
        return bytes(b)
    # a 4-byte field somewhere in the first part (widths, counts), rewritten
    i = rng.randrange(0, max(1, min(len(b), 400)) - 3)
    struct.pack_into("<I", b, i, rng.choice([0, 1, 31, 33, 64, 0x7FFFFFFF, 0xFFFFFFFF]))
    return bytes(b)

counts = {"zkey": [0, 0], "gnark": [0, 0], "wtns": [0, 0], "gw": [0, 0]}
for it in range(int(sys.argv[8])):
    b = mutate(zk, 12)
    k = ctypes.c_void_p()
    rc = L.g16_zkey_parse(b, len(b), rng.randrange(2), ctypes.byref(k))
    if rc == 0:
        L.g16_zkey_view_get(k, view)
        L.g16_zkey_free(k)
    counts["zkey"][rc == 0] += 1
    if it % 4 == 0:
        p2, v2 = (mutate(pk, None), vk) if rng.randrange(2) else (pk, mutate(vk, None))
        k = ctypes.c_void_p()
        rc = L.g16_gnark_key_parse(p2, len(p2), v2, len(v2), ctypes.byref(k))
        if rc == 0:
            L.g16_zkey_view_get(k, view)
            L.g16_zkey_free(k)
        counts["gnark"][rc == 0] += 1
    b = mutate(wtns, 12)
    n = ctypes.c_size_t()
    rc = L.g16_wtns_parse(b, len(b), None, 0, ctypes.byref(n))
    if rc == 0 and n.value < (1 << 20):
        out = ctypes.create_string_buffer(32 * max(1, n.value))
        rc = L.g16_wtns_parse(b, len(b), out, n.value, ctypes.byref(n))
    counts["wtns"][rc == 0] += 1
    b = mutate(gw, None)
    nw, nr = ctypes.c_size_t(), ctypes.c_size_t()
    rc = L.g16_gnark_witness_parse(b, len(b), None, 0, None, None, 0, ctypes.byref(nw), ctypes.byref(nr))
    if rc == 0 and nw.value < (1 << 20) and nr.value < (1 << 20):
        w = ctypes.create_string_buffer(32 * max(1, nw.value))
        a = ctypes.create_string_buffer(32 * max(1, nr.value))
        c = ctypes.create_string_buffer(32 * max(1, nr.value))
        rc = L.g16_gnark_witness_parse(b, len(b), w, nw.value, a, c, nr.value, ctypes.byref(nw), ctypes.byref(nr))
    counts["gw"][rc == 0] += 1
print(counts)
"""


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("fuzz")
    sc = S.SynthCircuit(seed=31, n_constraints=60, n_inputs=6, n_public=2)
    zk = sc.zkey(5)
    w = sc.witness(1)
    wt = S.wtns_bytes(w) if hasattr(S, "wtns_bytes") else None
    if wt is None:   # the library's writer
        import ctypes
        n = len(w) // 32
        ln = ctypes.c_size_t()
        S.check(S.lib().g16_wtns_write(w, n, None, 0, ctypes.byref(ln)))
        buf = ctypes.create_string_buffer(ln.value)
        S.check(S.lib().g16_wtns_write(w, n, buf, ln.value, ctypes.byref(ln)))
        wt = buf.raw[:ln.value]
    with gzip.open(os.path.join(GOLDEN, "gnark_toy_pk.dump.gz")) as f:
        pk = f.read()
    with gzip.open(os.path.join(GOLDEN, "gnark_toy_witness.bin.gz")) as f:
        gw = f.read()
    vk = bytes.fromhex(json.load(open(os.path.join(GOLDEN, "gnark_toy.json")))["vk.bin"])
    paths = []
    for name, data in (("zk", zk), ("pk", pk), ("vk", vk), ("wtns", wt), ("gw", gw)):
        p = d / name
        p.write_bytes(data)
        paths.append(str(p))
    return paths


@pytest.mark.parametrize("seed", [1, 2])
def test_readers_survive_malformed_input(inputs, seed):
    r = subprocess.run([sys.executable, "-c", FUZZ, ROOT] + inputs + [str(seed), "800"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, "a reader crashed (status %d): %s" % (r.returncode, r.stderr[-2000:])
    counts = eval(r.stdout.strip().splitlines()[-1])
    # most mutations are refused; the unmodified-looking ones may parse
    assert all(bad + ok > 0 for bad, ok in counts.values()), counts
