"""The reference work model that bench.py reports beside its own rooflines.

The MSM lines carry `work_model_roofline`: the reference's window size for the
m general scalars (crates/msm/src/lib.rs:160-172) and its product count.  The
figures for uniform scalars must reproduce the worked examples of the work
model: c = 13 at N = 2^16 with 15.4M Fq products, c = 16 at 2^20 with 182.5M.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def scalars(n, ones=0, zeros=0, seed=1):
    rng = np.random.default_rng(seed)
    v = np.zeros((n, 4), dtype=np.uint64)
    v[:, 0] = rng.integers(2, 2 ** 63, n, dtype=np.uint64)
    v[:ones, 0] = 1
    v[ones:ones + zeros, 0] = 0
    return v.tobytes()


def test_reference_window_size():
    assert bench.reference_window_size(1 << 16) == 13
    assert bench.reference_window_size(1 << 20) == 16
    assert bench.reference_window_size(1 << 22) == 16
    assert 3 <= bench.reference_window_size(1) <= 16


def test_work_model_examples():
    m16 = bench.msm_work_model(scalars(1 << 16), False)
    assert (m16["c"], m16["general_scalars"]) == (13, 1 << 16)
    assert m16["fq_products"] == 10 * (1 << 16) * 20 + 28 * 4096 * 20   # 15.4M
    m20 = bench.msm_work_model(scalars(1 << 20), False)
    assert m20["fq_products"] == 182_452_224
    g2 = bench.msm_work_model(scalars(1 << 10), True)
    assert g2["fq_products"] == 3 * bench.msm_work_model(scalars(1 << 10), False)["fq_products"]


def test_work_model_counts_zeros_and_ones():
    m = bench.msm_work_model(scalars(1000, ones=300, zeros=400), False)
    assert (m["ones"], m["zeros"], m["general_scalars"]) == (300, 400, 300)
    c = bench.reference_window_size(300)
    w, b = -(-255 // c), 1 << (c - 1)
    assert m["fq_products"] == 10 * 300 * w + 28 * b * w + 10 * 300


def test_reference_arm_prints_the_contract_line(tmp_path):
    # `bench.py --impl reference` runs on host cores only; its one JSON line carries the
    # keys the driver reads, on the same metric and config as the GPU arm
    import json
    import subprocess
    env = dict(os.environ, G16_BENCH_CACHE=str(tmp_path))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--constraints", "3000",
                        "--steps", "2", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "proofs/s" and d["unit"] == "proofs/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert (d["steps"], d["warmup"]) == (2, 1) and d["ms_per_step"] > 0
    assert d["scaling"] == "weak" and d["vs_baseline"] is None and d["data"] == "synthetic"
    assert d["config"]["n_constraints"] == 3000 and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["parity"]["pairing_checked"] == d["parity"]["of"] == 3 and d["parity"]["bit_exact_vs_oracle"] is True
