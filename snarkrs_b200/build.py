"""Build recipe for ``snarkrs_b200/libg16b200.so`` (sm_100a, in-tree).

Every translation unit is compiled by nvcc for ``sm_100a`` only
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``); host C++ goes through
nvcc's host compiler.  Objects land in ``snarkrs_b200/_build/``; the shared
library sits next to this file so it travels with the package.

Usage: ``python -m snarkrs_b200.build [--force] [--verbose]``.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libg16b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["host_bn254.cpp", "formats.cpp", "gnark.cpp", "synth.cpp", "msm.cu", "msm_noalloc.cu", "ntt.cu", "prover.cu", "batch.cu", "server.cpp", "pairing.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
# extra nvcc flags for experiments (e.g. -DACC_G2_MIN_BLOCKS=3); pass --force when they change
EXTRA = os.environ.get("G16_NVCC_EXTRA", "").split()


def _headers():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not _stale(obj, [path] + _headers()):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    cmd = [NVCC] + ARCH + COMMON + EXTRA + lang + ["-c", path, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
