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
    printf("%zu %u %u %zu\n", g16::MSM_RESULT_SLOT_BYTES, g16::MSM_REDUCE_LB_G1, g16::MSM_REDUCE_LB_G2,
           g16::MSM_RESULT_SLOT_COMPACT_BYTES);
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
        run.slot_bytes, run.lb_g1, run.lb_g2, run.compact_slot_bytes = map(int, out[0].split())
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


def test_compact_key_results_fit_the_readback_slot(plan):
    # a compact key reduces one bucket set per window (the standalone MSM's plan, aiming at
    # 32768 pieces), for every window width a tuning may set (8 to 20 bits)
    cases = [((255 + c - 1) // c, 1 << (c - 1), g2, 32768) for c in range(8, 21) for g2 in (0, 1)]
    results = plan(cases)
    assert plan.compact_slot_bytes == 128 * 1024
    for (_, _, g2, _), p in zip(cases, results):
        assert p["result_points"] * (256 if g2 else 128) <= plan.compact_slot_bytes


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


LAYOUT_PROBE = r"""
#include <cstdio>
#include <vector>
#include "msm.cuh"
int main() {
    printf("%u %u %u\n", g16::MSM_REDUCE_LB_G1, g16::MSM_REDUCE_LB_G2, g16::MSM_REDUCE_MAX_SEG);
    unsigned nseg, g2, sms, override_len;
    unsigned long long target;
    while (scanf("%u %u %llu %u %u", &nseg, &g2, &target, &sms, &override_len) == 5) {
        std::vector<uint32_t> B(nseg);
        for (auto& b : B) scanf("%u", &b);
        g16::MsmSpaceReduceLayout L = g16::msm_space_reduce_layout(B, g2 != 0, target, sms, override_len);
        printf("%llu %llu %llu %llu %u %u\n", (unsigned long long)L.K, (unsigned long long)L.blocks,
               (unsigned long long)L.block_points, (unsigned long long)L.result_points, L.max_hb, L.piece_len);
        for (size_t j = 0; j < B.size(); j++) {
            const g16::MsmReducePlan& p = L.plans[j];
            printf("%u %u %u %u %u %d %u %u %u %u %u\n", p.seg, p.lb, p.nb, p.hb, p.sets, p.direct ? 1 : 0,
                   L.key_start[j], L.block_start[j], L.out_block[j], L.out_set[j], p.set_terms());
        }
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def layout():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    import tempfile
    d = tempfile.mkdtemp(prefix="layout_probe")
    src, exe = os.path.join(d, "probe.cu"), os.path.join(d, "probe")
    open(src, "w").write(LAYOUT_PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, src], check=True, capture_output=True)

    def run(cases):
        text = "".join("%d %d %d %d %d %s\n" % (len(Bs), g2, target, sms, ovr, " ".join(map(str, Bs)))
                       for Bs, g2, target, sms, ovr in cases)
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
        run.lb_g1, run.lb_g2, run.max_seg = map(int, out[0].split())
        res, i = [], 1
        for Bs, *_ in cases:
            tot = dict(zip(("K", "blocks", "block_points", "result_points", "max_hb", "piece_len"),
                           map(int, out[i].split())))
            segs = [dict(zip(("seg", "lb", "nb", "hb", "sets", "direct", "key_start", "block_start", "out_block",
                              "out_set", "set_terms"), map(int, out[i + 1 + j].split()))) for j in range(len(Bs))]
            res.append((tot, segs))
            i += 1 + len(Bs)
        return res
    yield run
    shutil.rmtree(d, ignore_errors=True)


def test_batched_reduction_layout_matches_the_kernels(layout):
    # Random mixes of segments (the batched engine's spaces) laid out by
    # msm_space_reduce_layout, then the indexing of k_reduce_pieces_multi and
    # k_reduce_sets_multi replayed on that layout: every block finds its own
    # segment, reads only its segment's buckets, and writes only its own points;
    # every sets-kernel read and write stays inside its segment and the buffers.
    import random
    rng = random.Random(11)
    cases = []
    for _ in range(300):
        nseg = rng.randrange(1, 40)
        Bs = [1 << (rng.randrange(4, 22) - 1) for _ in range(nseg)]
        g2 = rng.randrange(2)
        target = rng.choice([0, 0, 0, 8192, 32768, 1 << rng.randrange(4, 18)])
        sms = rng.choice([148, 132, 1, 7])
        ovr = rng.choice([0, 0, 0, 0, 1, 2, 8, 32, 3, 64])
        cases.append((Bs, g2, target, sms, ovr))
    for (Bs, g2, target, sms, ovr), (tot, segs) in zip(cases, layout(cases)):
        LB = layout.lb_g2 if g2 else layout.lb_g1   # the kernels' template argument
        assert tot["K"] == sum(Bs)
        if ovr in (1, 2, 4, 8, 16, 32):
            assert tot["piece_len"] == ovr
        k = b = bp = rp = 0
        for B, s in zip(Bs, segs):
            assert s["lb"] == LB and s["sets"] == 1 and s["direct"] == 0
            assert (s["key_start"], s["block_start"], s["out_block"], s["out_set"]) == (k, b, bp, rp)
            pieces = B // s["seg"]
            assert pieces * s["seg"] == B and 1 <= s["seg"] <= layout.max_seg
            nb, hb = s["nb"], s["hb"]
            assert nb >= 1 and (nb << LB) >= pieces and ((nb - 1) << LB) < pieces and (1 << hb) == nb
            # k_reduce_pieces_multi: block jb < nb of this segment reads buckets
            # key_start + p*seg + i (p*seg < B) and writes out_block + jb*(LB+2) + [0, LB+1]
            last_write = s["out_block"] + (nb - 1) * (LB + 2) + LB + 1
            assert last_write < bp + nb * (LB + 2) <= tot["block_points"]
            # k_reduce_sets_multi: term o < LB+1+hb reads out_block + j*(LB+2) + min(o, LB+1), j < nb,
            # and writes out_set + o
            assert s["set_terms"] == LB + 1 + hb
            assert s["out_set"] + LB + hb < rp + s["set_terms"] <= tot["result_points"]
            k += B
            b += nb
            bp += nb * (LB + 2)
            rp += s["set_terms"]
        assert (k, b, bp, rp) == (tot["K"], tot["blocks"], tot["block_points"], tot["result_points"])
        assert tot["max_hb"] == max(s["hb"] for s in segs)
        # a block finds its segment by the last block_start <= block (strictly increasing)
        starts = [s["block_start"] for s in segs]
        assert all(x < y for x, y in zip(starts, starts[1:]))


def _plan_probe(defines):
    """The plan probe compiled with extra -D flags (another reduction block size)."""
    import tempfile
    d = tempfile.mkdtemp(prefix="plan_probe_d")
    src, exe = os.path.join(d, "probe.cu"), os.path.join(d, "probe")
    open(src, "w").write(PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O1"] + defines + ["-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, src], check=True, capture_output=True)

    def run(cases):
        text = "\n".join("%d %d %d %d" % c for c in cases) + "\n"
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
        keys = ("seg", "lb", "nb", "hb", "direct", "set_terms", "block_points", "result_points")
        return [dict(zip(keys, map(int, l.split()))) for l in out[1:] if l.strip()]
    return run, d


def _emulate_reduction(S, sets, B, p):
    """k_reduce_pieces, k_reduce_sets and the host's set_sum (msm.cu) on integers standing
    in for points (addition is +, doubling is *2), step by step as the kernels index them.
    Returns each set's sum_b (b + 1) S_b as the device and host would form it."""
    LB, seg, nb, hb = p["lb"], p["seg"], p["nb"], p["hb"]
    N = 1 << LB
    weighted = seg > 1
    terms = LB + 2
    blocks_out = [0] * (sets * nb * terms)
    for st in range(sets):
        for jb in range(nb):
            run, tot = [0] * N, [0] * N
            for t in range(N):
                pc = jb * N + t
                if pc * seg < B:
                    g0 = st * B + pc * seg
                    for i in range(seg - 1, -1, -1):
                        run[t] += S[g0 + i]
                        if weighted:
                            tot[t] += run[t]
            s_run, s_tot = list(run), list(tot)
            lg = [0 if t == 0 else t.bit_length() - 1 for t in range(N)]
            for k in range(1, LB + 1):
                h = N >> k
                r_run, r_tot = list(s_run), list(s_tot)   # a step reads the state the barrier left
                for t in range(N):
                    if t < h:
                        run[t] = run[t] + r_run[t + h]
                        s_run[t] = run[t]
                    elif t < 2 * h:
                        if weighted:
                            tot[t] = r_tot[t - h] + r_tot[t]
                            s_tot[t - h] = tot[t]
                    else:
                        hs, s = 1 << lg[t], 1 << (k - (LB - lg[t]) - 1)
                        o = t - hs
                        if (o & (2 * s - 1)) == 0 and o + s < hs:
                            run[t] = run[t] + r_run[t + s]
                            s_run[t] = run[t]
            o0 = (st * nb + jb) * terms
            for t in range(N):
                if t == 0:
                    if not weighted:
                        blocks_out[o0] = run[0]
                    blocks_out[o0 + LB + 1] = run[0]
                elif t & (t - 1) == 0:
                    blocks_out[o0 + 1 + lg[t]] = run[t]
                    if t == 1 and weighted:
                        blocks_out[o0] = tot[1]
    sums = []
    for st in range(sets):
        base = st * nb * terms
        if p["direct"]:
            T, G, Gb = 0, [0] * LB, [0] * hb
            for j in range(nb):
                o = base + j * terms
                T += blocks_out[o]
                for i in range(LB):
                    G[i] += blocks_out[o + 1 + i]
                for i in range(hb):
                    if (j >> i) & 1:
                        Gb[i] += blocks_out[o + LB + 1]
        else:   # k_reduce_sets: term o of the set over its nb blocks
            res = []
            for o in range(LB + 1 + hb):
                acc = 0
                for j in range(nb):
                    if o <= LB:
                        acc += blocks_out[base + j * terms + o]
                    elif (j >> (o - LB - 1)) & 1:
                        acc += blocks_out[base + j * terms + LB + 1]
                res.append(acc)
            T, G, Gb = res[0], res[1:1 + LB], res[LB + 1:]
        acc = 0
        for i in range(hb - 1, -1, -1):
            acc = 2 * acc + Gb[i]
        for j in range(LB - 1, -1, -1):
            acc = 2 * acc + G[j]
        s = seg
        while s > 1:
            acc *= 2
            s >>= 1
        sums.append(acc + T)
    return sums


@pytest.mark.parametrize("defines", [[], ["-DG16_REDUCE_LB_G1=7", "-DG16_REDUCE_LB_G2=6"]],
                         ids=["blocks-of-2^8", "blocks-of-2^7-and-2^6"])
def test_reduction_algebra_by_integer_emulation(defines):
    # the pieces kernel's running sums, halvings and per-bit trees, the sets kernel and the
    # host's combination give sum_b (b + 1) S_b for every plan shape: direct and summed on
    # the device, weighted (seg > 1) and not, one or several sets
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    import random
    run, d = _plan_probe(defines)
    try:
        rng = random.Random(5)
        cases = []
        for B in (1, 2, 8, 64, 256, 1024, 4096):
            for sets in (1, 2, 3):
                for g2 in (0, 1):
                    for target in (1, 16, 256, 8192, 32768):
                        cases.append((sets, B, g2, target))
        shapes = set()
        for (sets, B, g2, target), p in zip(cases, run(cases)):
            shape = (sets, B, p["seg"], p["nb"], p["direct"], p["lb"])
            if shape in shapes:
                continue
            shapes.add(shape)
            S = [rng.randrange(1, 1 << 20) for _ in range(sets * B)]
            want = [sum((b + 1) * S[st * B + b] for b in range(B)) for st in range(sets)]
            assert _emulate_reduction(S, sets, B, p) == want, (sets, B, g2, target, p)
        assert any(s[4] == 1 for s in shapes) and any(s[4] == 0 for s in shapes)
        assert any(s[2] > 1 for s in shapes) and any(s[2] == 1 for s in shapes)
    finally:
        shutil.rmtree(d, ignore_errors=True)
