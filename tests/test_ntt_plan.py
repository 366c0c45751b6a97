"""Host-side check of the NTT kernels' indexing (snarkrs_b200/csrc/ntt.cu) on the CPU.

The pass plan comes from the product's own host code (ntt_inner_k and
ntt_outer_passes in ntt.cuh, compiled here by nvcc for the CPU).  The kernels'
index arithmetic, restated here line for line from ntt.cu (the GPU parity tests
check the CUDA code itself), is then replayed on integers mod r: run_stage's butterfly
pairs and twiddle positions, ntt_pass_tile's tile-to-global mapping, the fused
middle's DIF stages, coset multiply and DIT stages, and the launch order of
ntt_intt_coset_ntt and ntt_h_pipeline (including the H = A*B - C join on the
last pass).  Every valid tiling at small sizes must give the oracle's
intt_coset_ntt, and the pipeline the oracle's H."""
import os
import random
import shutil
import subprocess

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
R = O.R_MOD

PROBE = r"""
#include <cstdio>
#include "ntt.cuh"
int main() {
    unsigned tile_log, outer_log_l, log_n;
    while (scanf("%u %u %u", &tile_log, &outer_log_l, &log_n) == 3) {
        g16::NttTiling t;
        t.tile_log = tile_log;
        t.outer_log_l = outer_log_l;
        if (!g16::ntt_tiling_valid(t)) { printf("invalid\n"); continue; }
        const unsigned k0 = g16::ntt_inner_k(t, log_n);
        auto passes = g16::ntt_outer_passes(t, log_n, k0);
        printf("%u %zu", k0, passes.size());
        for (auto& p : passes) printf(" %u %u %u", p.s_lo, p.k, p.log_L);
        printf("\n");
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def plans():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    import tempfile
    d = tempfile.mkdtemp(prefix="ntt_probe")
    src, exe = os.path.join(d, "probe.cu"), os.path.join(d, "probe")
    open(src, "w").write(PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, src], check=True, capture_output=True)

    def run(cases):
        text = "".join("%d %d %d\n" % c for c in cases)
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
        res = []
        for line in out[:len(cases)]:
            if line == "invalid":
                res.append(None)
                continue
            v = list(map(int, line.split()))
            res.append((v[0], [tuple(v[2 + 3 * i:5 + 3 * i]) for i in range(v[1])]))
        return res
    yield run
    shutil.rmtree(d, ignore_errors=True)


def run_stage(dif, sm, j, s_lo, log_L, lo0, log_n, half_tile, tw):
    L = 1 << log_L
    s = s_lo + j
    jmask = (1 << j) - 1
    for q in range(half_tile):   # one butterfly per q; the pairs of a stage are disjoint
        l, mq = q & (L - 1), q >> log_L
        mid_a = ((mq >> j) << (j + 1)) | (mq & jmask)
        ea = (mid_a << log_L) | l
        eb = ea + (1 << (j + log_L))
        pos = ((mid_a & jmask) << s_lo) | (lo0 + l)
        a, b = sm[ea], sm[eb]
        w = tw[pos << (log_n - s - 1)]
        if dif:
            d = a - b
            a, b = a + b, (d * w if pos else d)
        else:
            t = b * w if pos else b
            a, b = a + t, a - t
        sm[ea], sm[eb] = a % R, b % R


def pass_tile(dif, data, bx, log_n, s_lo, k, log_L, tw, join=None):
    L = 1 << log_L
    tile = (1 << k) << log_L
    bph = s_lo - log_L
    assert bph >= 0
    hi, lo0 = bx >> bph, (bx & ((1 << bph) - 1)) << log_L
    gi = [(hi << (s_lo + k)) | ((e >> log_L) << s_lo) | (lo0 + (e & (L - 1))) for e in range(tile)]
    sm = [data[g] for g in gi]
    for jj in range(k):
        run_stage(dif, sm, k - 1 - jj if dif else jj, s_lo, log_L, lo0, log_n, tile // 2, tw)
    for e, g in enumerate(gi):
        if join:
            ja, jb, jo = join
            jo[g] = (ja[g] * jb[g] - sm[e]) % R
        else:
            data[g] = sm[e]


def mid_tile(data, bx, log_n, k, tw, tw_inv, coset, join=None):
    tile = 1 << k
    base = bx << k
    sm = data[base:base + tile]
    for j in range(k - 1, -1, -1):
        run_stage(True, sm, j, 0, 0, 0, log_n, tile // 2, tw_inv)
    sm = [(x * coset[base + e]) % R for e, x in enumerate(sm)]
    for j in range(k):
        run_stage(False, sm, j, 0, 0, 0, log_n, tile // 2, tw)
    for e in range(tile):
        if join:
            ja, jb, jo = join
            jo[base + e] = (ja[base + e] * jb[base + e] - sm[e]) % R
        else:
            data[base + e] = sm[e]


def tables(log_n):
    n = 1 << log_n
    w = O.from_mont(O.domain_root(log_n))
    shift = O.from_mont(O.domain_root(log_n + 1))
    wi, ninv = pow(w, R - 2, R), pow(n, R - 2, R)
    tw = [pow(w, i, R) for i in range(n // 2)]
    tw_inv = [pow(wi, i, R) for i in range(n // 2)]
    coset = [0] * n
    for i in range(n):   # k_powers with bitrev_log = log_n: coset[bitrev(i)] = shift^i / n
        coset[int(format(i, "0%db" % log_n)[::-1], 2) if log_n else 0] = ninv * pow(shift, i, R) % R
    return tw, tw_inv, coset


def grid(n, tile):
    return range(n // tile)


def emulate_intt_coset_ntt(plan, log_n, data, tabs):
    k0, outer = plan
    tw, tw_inv, coset = tabs
    n = 1 << log_n
    data = list(data)
    for s_lo, k, log_L in reversed(outer):
        for bx in grid(n, (1 << k) << log_L):
            pass_tile(True, data, bx, log_n, s_lo, k, log_L, tw_inv)
    for bx in grid(n, 1 << k0):
        mid_tile(data, bx, log_n, k0, tw, tw_inv, coset)
    for s_lo, k, log_L in outer:
        for bx in grid(n, (1 << k) << log_L):
            pass_tile(False, data, bx, log_n, s_lo, k, log_L, tw)
    return data


def emulate_h_pipeline(plan, log_n, a, b, c, tabs):
    """ntt_h_pipeline's launches in order: inverse passes of A, B, C; the middle (of A, B
    and C, or of A and B then C with the join when there are no outer passes); forward
    passes, the last one of A and B, then of C with h = A*B - C."""
    k0, outer = plan
    tw, tw_inv, coset = tabs
    n = 1 << log_n
    a, b, c, h = list(a), list(b), list(c), [0] * n
    for s_lo, k, log_L in reversed(outer):
        for v in (a, b, c):
            for bx in grid(n, (1 << k) << log_L):
                pass_tile(True, v, bx, log_n, s_lo, k, log_L, tw_inv)
    if not outer:
        for v in (a, b):
            for bx in grid(n, 1 << k0):
                mid_tile(v, bx, log_n, k0, tw, tw_inv, coset)
        for bx in grid(n, 1 << k0):
            mid_tile(c, bx, log_n, k0, tw, tw_inv, coset, join=(a, b, h))
        return h
    for v in (a, b, c):
        for bx in grid(n, 1 << k0):
            mid_tile(v, bx, log_n, k0, tw, tw_inv, coset)
    for s_lo, k, log_L in outer[:-1]:
        for v in (a, b, c):
            for bx in grid(n, (1 << k) << log_L):
                pass_tile(False, v, bx, log_n, s_lo, k, log_L, tw)
    s_lo, k, log_L = outer[-1]
    for v in (a, b):
        for bx in grid(n, (1 << k) << log_L):
            pass_tile(False, v, bx, log_n, s_lo, k, log_L, tw)
    for bx in grid(n, (1 << k) << log_L):
        pass_tile(False, c, bx, log_n, s_lo, k, log_L, tw, join=(a, b, h))
    return h


def oracle_icn(log_n, data):
    raw = b"".join(O.to_bytes(O.to_mont(x)) for x in data)
    out = O.ntt(log_n, O.NTT_INTT_COSET_NTT, raw)
    return [O.from_mont(O.from_bytes(out[32 * i:32 * i + 32])) for i in range(1 << log_n)]


def test_every_tiling_gives_the_oracle_intt_coset_ntt(plans):
    # tiles small enough that sizes up to 2^9 take several outer passes, including the
    # uneven splits and the narrowed columns (log_L < outer_log_l) of the lowest pass
    cases = [(t, l, n) for t in range(1, 7) for l in range(0, 6) for n in range(1, 10)]
    rng = random.Random(3)
    checked = 0
    for (t, l, log_n), plan in zip(cases, plans(cases)):
        assert (plan is None) == (not (2 <= t <= 12 and l < t and l <= 4))
        if plan is None:
            continue
        k0, outer = plan
        # the plan covers every stage once, in order, within the tile's rows
        s = k0
        for s_lo, k, log_L in outer:
            assert s_lo == s and 1 <= k <= t - l and log_L == min(l, s_lo)
            s += k
        assert s == log_n and k0 == min(log_n, t)
        data = [rng.randrange(R) for _ in range(1 << log_n)]
        tabs = tables(log_n)
        assert emulate_intt_coset_ntt(plan, log_n, data, tabs) == oracle_icn(log_n, data), (t, l, log_n)
        checked += 1
    assert checked > 100


def test_h_pipeline_gives_the_oracle_h(plans):
    cases = [(t, l, n) for t, l in ((2, 0), (2, 1), (3, 1), (4, 2), (5, 4), (11, 2)) for n in (1, 2, 5, 8)]
    rng = random.Random(4)
    for (t, l, log_n), plan in zip(cases, plans(cases)):
        n = 1 << log_n
        a, b, c = ([rng.randrange(R) for _ in range(n)] for _ in range(3))
        tabs = tables(log_n)
        A, B, C = oracle_icn(log_n, a), oracle_icn(log_n, b), oracle_icn(log_n, c)
        want = [(x * y - z) % R for x, y, z in zip(A, B, C)]
        assert emulate_h_pipeline(plan, log_n, a, b, c, tabs) == want, (t, l, log_n)


BATCH_PROBE = r"""
#include <cstdio>
#include <vector>
#include "ntt.cuh"
int main() {
    unsigned items;
    while (scanf("%u", &items) == 1) {
        std::vector<uint32_t> logs(items);
        std::vector<g16::NttTiling> tl(items);
        for (unsigned i = 0; i < items; i++) scanf("%u %u %u", &logs[i], &tl[i].tile_log, &tl[i].outer_log_l);
        auto phases = g16::ntt_batch_plan(logs, tl);
        printf("%zu\n", phases.size());
        for (auto& ph : phases) {
            printf("%d %zu", ph.kind, ph.jobs.size());
            for (auto& j : ph.jobs)
                printf(" %u %d %d %u %u %u %d", j.item, j.vec, j.kind, j.pass.s_lo, j.pass.k, j.pass.log_L, j.join ? 1 : 0);
            printf("\n");
        }
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def batch_plans():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    import tempfile
    d = tempfile.mkdtemp(prefix="ntt_batch_probe")
    src, exe = os.path.join(d, "probe.cu"), os.path.join(d, "probe")
    open(src, "w").write(BATCH_PROBE)
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "snarkrs_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), "-o", exe, src], check=True, capture_output=True)

    def run(batches):
        text = "".join("%d %s\n" % (len(b), " ".join("%d %d %d" % x for x in b)) for b in batches)
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
        res, i = [], 0
        for _ in batches:
            nph = int(out[i])
            phases = []
            for line in out[i + 1:i + 1 + nph]:
                v = list(map(int, line.split()))
                jobs = [tuple(v[2 + 7 * j:9 + 7 * j]) for j in range(v[1])]
                phases.append((v[0], jobs))
            res.append(phases)
            i += 1 + nph
        return res
    yield run
    shutil.rmtree(d, ignore_errors=True)


def test_batched_h_pipelines_give_the_oracle_h(batch_plans):
    # several items of different sizes and tilings in one batch (ntt_batch_plan), the
    # phases run in order; the jobs of a phase run side by side on the GPU, so no job
    # may read a vector that another job of its phase writes
    rng = random.Random(9)
    tilings = [(2, 0), (2, 1), (3, 1), (4, 2), (5, 4), (11, 2), (3, 0)]
    batches = []
    for _ in range(25):
        batches.append([(rng.randrange(1, 9),) + rng.choice(tilings) for _ in range(rng.randrange(1, 5))])
    for batch, phases in zip(batches, batch_plans(batches)):
        vecs, want, tabs = [], [], []
        for log_n, t, l in batch:
            n = 1 << log_n
            a, b, c = ([rng.randrange(R) for _ in range(n)] for _ in range(3))
            A, B, C = oracle_icn(log_n, a), oracle_icn(log_n, b), oracle_icn(log_n, c)
            want.append([(x * y - z) % R for x, y, z in zip(A, B, C)])
            vecs.append([a, b, c, [0] * n])
            tabs.append(tables(log_n))
        for kind, jobs in phases:
            for item, vec, jkind, s_lo, k, log_L, join in jobs:
                assert jkind == kind
                log_n = batch[item][0]
                n = 1 << log_n
                tw, tw_inv, coset = tabs[item]
                v = vecs[item]
                jn = (v[0], v[1], v[3]) if join else None
                if kind == 2:
                    for bx in grid(n, 1 << k):
                        mid_tile(v[vec], bx, log_n, k, tw, tw_inv, coset, join=jn)
                else:
                    for bx in grid(n, (1 << k) << log_L):
                        pass_tile(kind == 0, v[vec], bx, log_n, s_lo, k, log_L, tw_inv if kind == 0 else tw, join=jn)
            # a job may rewrite its own vector; no job touches what another writes
            per_job = [((it, 3 if jn_ else vc), {(it, vc)} | ({(it, 0), (it, 1)} if jn_ else set()))
                       for it, vc, _, _, _, _, jn_ in jobs]
            for i, (w, _) in enumerate(per_job):
                for j, (_, r) in enumerate(per_job):
                    assert i == j or w not in r, (batch, kind, jobs[i], jobs[j])
        for item in range(len(batch)):
            assert vecs[item][3] == want[item], (batch, item)
