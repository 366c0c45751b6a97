"""Host-side check of the MSM bucket-reduction plan (msm_reduce_plan in
snarkrs_b200/csrc/msm.cuh), compiled here by nvcc for the CPU.

For every window width the prover and the standalone MSM can use, over G1 and
G2 and both piece targets, the plan must cover every bucket exactly once
(pieces x seg = B, blocks x 2^lb >= pieces), keep seg a power of two no larger
than 32, take the direct path only for at most two blocks in all, and give a
prover MSM result that fits the prover's readback slot per MSM (MSM_RESULT_SLOT_BYTES).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
#include <cstdio>
#include "msm.cuh"
int main() {
    printf("%zu %u %u\n", g16::MSM_RESULT_SLOT_BYTES, g16::MSM_REDUCE_LB_G1, g16::MSM_REDUCE_LB_G2);
    unsigned sets, B, g2;
    unsigned long long target;
    while (scanf("%u %u %u %llu", &sets, &B, &g2, &target) == 4) {
        g16::MsmReducePlan p = g16::msm_reduce_plan(sets, B, g2 != 0, target);
        printf("%u %u %u %u %d %u %zu %zu\n", p.seg, p.lb, p.nb, p.hb, p.direct ? 1 : 0, p.set_terms(),
               p.block_points(), p.result_points());
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def plan():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    import tempfile
    d = tempfile.mkdtemp(prefix="plan_probe")
    src, exe = os.path.join(d, "probe.cu"), os.path.join(d, "probe")
    open(src, "w").write(PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, src], check=True, capture_output=True)

    def run(cases):
        text = "\n".join("%d %d %d %d" % c for c in cases) + "\n"
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
        run.slot_bytes, run.lb_g1, run.lb_g2 = map(int, out[0].split())
        keys = ("seg", "lb", "nb", "hb", "direct", "set_terms", "block_points", "result_points")
        return [dict(zip(keys, map(int, l.split()))) for l in out[1:] if l.strip()]
    yield run
    shutil.rmtree(d, ignore_errors=True)


def test_plans_cover_every_bucket(plan):
    cases = []
    for c in range(1, 23):
        B = 1 << (c - 1)
        for sets in (1, 2, 3, (255 + c - 1) // c):
            for g2 in (0, 1):
                for target in (8192, 32768):
                    cases.append((sets, B, g2, target))
    for (sets, B, g2, target), p in zip(cases, plan(cases)):
        seg, lb, nb = p["seg"], p["lb"], p["nb"]
        assert lb == (plan.lb_g2 if g2 else plan.lb_g1)
        assert seg & (seg - 1) == 0 and 1 <= seg <= 32 and seg <= B
        pieces = B // seg
        assert pieces * seg == B
        assert nb & (nb - 1) == 0 and nb << lb >= pieces and (nb - 1) << lb < pieces
        assert (1 << p["hb"]) == nb
        assert p["direct"] == (sets * nb <= 2)
        if seg < 32 and seg < B:
            assert sets * B // seg <= target      # seg stops growing once the target is met
        if seg > 1:
            assert sets * B // (seg // 2) > target
        assert p["block_points"] == sets * nb * (lb + 2)
        terms = nb * (lb + 2) if p["direct"] else lb + 1 + p["hb"]
        assert p["set_terms"] == terms and p["result_points"] == sets * terms


def test_prover_results_fit_the_readback_slot(plan):
    # the prover reads each MSM's result into a pinned slot of MSM_RESULT_SLOT_BYTES; its
    # windows share one bucket set, with c up to 22 and either target (the H MSM uses the
    # larger one)
    cases = [(1, 1 << (c - 1), g2, t) for c in range(1, 23) for g2 in (0, 1) for t in (8192, 32768)]
    results = plan(cases)
    assert plan.slot_bytes == 32 * 256
    # a block of 2^lb threads at ~250 registers: at most 256 threads fit an SM's register file
    assert 1 <= plan.lb_g1 <= 8 and 1 <= plan.lb_g2 <= 8
    for (_, _, g2, _), p in zip(cases, results):
        assert p["result_points"] * (256 if g2 else 128) <= plan.slot_bytes
