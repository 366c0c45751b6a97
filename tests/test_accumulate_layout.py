"""The MSM accumulate's chunking and partial-sum layout (msm.cu: chunk_len, k_nseg,
accumulate_chunks, k_fat_merge_jobs/_final, k_bucket_sums), restated line for
line on Python integers (a point becomes the integer it stands for, an addition
a +).  For skewed bucket sizes -- empty buckets, a bucket holding most entries
(a witness full of ones), single entries -- every chunk's partial sum lands in
its own slot of its bucket's range, every slot is written once, the fat-bucket
jobs and the bucket sums give each bucket the sum of its entries, and the chunk
length keeps the thread count within its cap.  The GPU parity tests check the
CUDA code itself."""
import random

ACC_THREADS = 1 << 19
FAT_PARTIALS, FAT_JOBS, FAT_JOB_MIN = 16, 64, 128


def chunk_len(M, K, L_min, wave):
    L = (M + ACC_THREADS - 1) // ACC_THREADS
    per_bucket = (M + 4 * K - 1) // (4 * K)
    L = max(L, per_bucket, L_min)
    if wave and M:
        chunks = (M + L - 1) // L
        waves = (chunks + wave - 1) // wave
        if waves > 1:
            L2 = (M + (waves - 1) * wave - 1) // ((waves - 1) * wave)
            if 20 * (waves - 1) * L2 < 19 * waves * L:
                L = L2
    return L


def fat_job_len(ns):
    return max(FAT_JOB_MIN, (ns + FAT_JOBS - 1) // FAT_JOBS)


def layout_and_sums(sizes, values, L):
    Ks = len(sizes)
    offsets = [0]
    for s in sizes:
        offsets.append(offsets[-1] + s)
    M = offsets[-1]
    # k_nseg: partials per bucket; seg_base is their exclusive scan
    nseg = [((hi - 1) // L - lo // L + 1) if hi > lo else 0 for lo, hi in zip(offsets, offsets[1:])]
    seg_base = [0]
    for n in nseg:
        seg_base.append(seg_base[-1] + n)
    partials = [None] * seg_base[-1]

    def store(g, t, acc):
        slot = seg_base[g] + (t - offsets[g] // L)
        assert seg_base[g] <= slot < seg_base[g] + nseg[g], (g, t)
        assert partials[slot] is None, "a slot written twice"
        partials[slot] = acc

    for t in range((M + L - 1) // L):   # accumulate_chunks, one thread per chunk
        start, end = t * L, min(t * L + L, M)
        lo, hi = 0, Ks
        while hi - lo > 1:
            mid = (lo + hi) >> 1
            if offsets[mid] <= start:
                lo = mid
            else:
                hi = mid
        g, nxt, acc = lo, offsets[lo + 1], 0
        for k in range(start, end):
            if k == nxt:
                store(g, t, acc)
                acc = 0
                g += 1
                nxt = offsets[g + 1]
                while nxt <= k:
                    g += 1
                    nxt = offsets[g + 1]
            acc += values[k]
        store(g, t, acc)
    assert None not in partials, "a partial slot no chunk wrote"
    # fat buckets: FAT_JOBS jobs of J partials folded into each job's first slot, then
    # the job results (slots base + t J, one thread each) into the first slot
    for g in range(Ks):
        ns, base = nseg[g], seg_base[g]
        if ns <= FAT_PARTIALS:
            continue
        J = fat_job_len(ns)
        assert FAT_JOBS * J >= ns
        for j in range(FAT_JOBS):
            a = j * J
            if a < ns:
                partials[base + a] = sum(partials[base + a:base + min(a + J, ns)])
        partials[base] = sum(partials[base + t * J] for t in range(64) if t * J < ns)
    # k_bucket_sums
    return [partials[seg_base[g]] if nseg[g] > FAT_PARTIALS else sum(partials[seg_base[g]:seg_base[g] + nseg[g]])
            for g in range(Ks)], offsets


def test_chunk_partials_fold_back_to_each_bucket():
    rng = random.Random(21)
    for trial in range(48):
        K = rng.choice([1, 2, 7, 64, 512, 2048])
        kind = trial % 4
        if kind == 0:     # uniform
            sizes = [rng.randrange(0, 12) for _ in range(K)]
        elif kind == 1:   # a witness of ones: one bucket holds most entries
            sizes = [rng.randrange(0, 3) for _ in range(K)]
            sizes[rng.randrange(K)] += rng.randrange(2000, 12000)
        elif kind == 2:   # mostly empty
            sizes = [rng.choice([0, 0, 0, 0, 1, 30]) for _ in range(K)]
        else:             # a few giant buckets
            sizes = [rng.choice([0, 0, 0, 1, 3000]) for _ in range(min(K, 64))]
        sizes.append(rng.randrange(0, 50))   # the constant-work sink bucket, accumulated, never reduced
        M = sum(sizes)
        if M == 0:
            continue
        values = [rng.randrange(1, 1 << 30) for _ in range(M)]
        L = chunk_len(M, K, 16, rng.choice([0, 148 * 512, 148]))
        assert L >= 16 and (M + L - 1) // L <= max(ACC_THREADS, 1)
        sums, offsets = layout_and_sums(sizes, values, L)
        for g in range(len(sizes)):
            assert sums[g] == sum(values[offsets[g]:offsets[g + 1]]), (trial, g)


def test_chunk_len_cases():
    # the device's choice: at least L_min, about M / (4 K) or more, and wave fitting
    # only for a gain of 5% or more
    assert chunk_len(1000, 1 << 16, 16, 0) == 16
    assert chunk_len(1 << 26, 1 << 16, 16, 0) == 256          # M / (4K)
    assert chunk_len(1 << 30, 1 << 20, 16, 0) == 2048         # the thread cap, 2^19 threads
    wave = 148 * 512                                          # one 512-thread block per SM
    M = int(2.4 * wave * 16)                                  # 2.4 waves of 16 lose to 2 waves of 20
    assert chunk_len(M, 1 << 20, 16, wave) == 20
    M = int(2.97 * wave * 16)                                 # 3 waves of 16 against 2 of 24: kept
    assert chunk_len(M, 1 << 20, 16, wave) == 16
