"""Regenerate the golden fixtures in this directory from the reference tree.

Reads (never writes) the reference checkout whose path is given as the first
argument or in ``G16_REFERENCE`` (there is no default), and writes:

* ``reference_constants.json`` -- the constants the reference's own tests pin:
  the ffjavascript domain roots for 2^28 and 2^4
  (crates/groth16/src/prove.rs:549-563), the BN254 moduli and CIOS n0 values
  (crates/gpu-layout/src/lib.rs:80-113), R mod r computed independently of
  arkworks (crates/gpu-layout/src/lib.rs:526-540) and the trace blinders
  (crates/groth16/src/trace.rs:43-47).  Each is extracted from the source text
  by a regular expression, not retyped.
* ``gnark_toy.json`` -- the committed gnark v0.14 toy fixture
  (test-support/gnark/toy/{vk.bin,proof.bin,public.bin}) as hex: a real
  gnark-produced Groth16 proof that an independent pairing must accept.
* ``gnark_toy_pk.dump.gz`` and ``gnark_toy_witness.bin.gz`` -- the same
  fixture's proving-key dump (``ProvingKey.WriteDump``) and witness dump (W,
  A.w and B.w), gzip-compressed byte for byte: the gnark key the rows path
  proves with, under gnark's bit-reversed H basis.

Run: ``python tests/golden/make_golden.py <reference checkout>``.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("G16_REFERENCE")
if __name__ == "__main__" and not REF:
    sys.exit("usage: make_golden.py <reference checkout> (or set G16_REFERENCE)")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def limbs32(text, name):
    m = re.search(r"pub const %s: \[u32; LIMBS\] = \[(.*?)\];" % name, text, re.S)
    if not m:
        m = re.search(r"const %s: \[u32; LIMBS\] = \[(.*?)\];" % name, text, re.S)
    words = [int(w.replace("_", ""), 16) for w in re.findall(r"0x[0-9a-f_]+", m.group(1))]
    assert len(words) == 8, name
    return sum(w << (32 * i) for i, w in enumerate(words))


def u32_const(text, name):
    m = re.search(r"pub const %s: u32 = (0x[0-9a-f_]+);" % name, text)
    return int(m.group(1).replace("_", ""), 16)


def main():
    layout = read("crates/gpu-layout/src/lib.rs")
    prove = read("crates/groth16/src/prove.rs")
    trace = read("crates/groth16/src/trace.rs")
    roots = re.findall(r'w\("(\d+)"\)', prove)
    assert len(roots) >= 2, roots
    tr = int(re.search(r"pub const TRACE_R: u64 = (0x[0-9a-f_]+);", trace).group(1).replace("_", ""), 16)
    ts = int(re.search(r"pub const TRACE_S: u64 = (0x[0-9a-f_]+);", trace).group(1).replace("_", ""), 16)
    consts = {
        "source": "zemse/snarkrs test constants, extracted by tests/golden/make_golden.py",
        "domain_root_2_28": roots[0],
        "domain_root_2_4": roots[1],
        "fr_modulus": str(limbs32(layout, "FR_MODULUS")),
        "fq_modulus": str(limbs32(layout, "FQ_MODULUS")),
        "fr_n0_u32": u32_const(layout, "FR_N0"),
        "fq_n0_u32": u32_const(layout, "FQ_N0"),
        "fr_r_mod_r": str(limbs32(layout, "FR_R_MOD_N")),
        "trace_r": tr,
        "trace_s": ts,
    }
    with open(os.path.join(HERE, "reference_constants.json"), "w") as f:
        json.dump(consts, f, indent=1)
        f.write("\n")

    toy = {}
    for name in ("vk.bin", "proof.bin", "public.bin"):
        with open(os.path.join(REF, "test-support/gnark/toy", name), "rb") as f:
            toy[name] = f.read().hex()
    toy["source"] = "test-support/gnark/toy (gnark v0.14.0 WriteTo / WriteRawTo), hex"
    with open(os.path.join(HERE, "gnark_toy.json"), "w") as f:
        json.dump(toy, f, indent=1)
        f.write("\n")
    import gzip
    for name, out in (("pk.dump", "gnark_toy_pk.dump.gz"), ("witness.bin", "gnark_toy_witness.bin.gz")):
        with open(os.path.join(REF, "test-support/gnark/toy", name), "rb") as f:
            data = f.read()
        with gzip.GzipFile(os.path.join(HERE, out), "wb", mtime=0) as g:
            g.write(data)
    print("wrote reference_constants.json, gnark_toy.json and the gnark toy dumps", file=sys.stderr)


if __name__ == "__main__":
    main()
