#!/usr/bin/env python
"""Groth16 / BN254 prove throughput on B200 (proofs/s), one JSON line.

Workload: one plain Groth16 prove of a seeded synthetic R1CS with 1,100,000
constraints (domain 2^21, 1,100,257 wires), the witness-value mix of the
configs (about 60% in {0,1}, 20% below 2^32, 20% uniform), a key written from
seeded toxic waste, seeded blinders r and s.  A step is one full proof:
stages 0-11 (gather, iNTT -> coset -> NTT of A, B, C, H = A*B - C, the five
MSMs, blinding and assembly).  Every step proves a different witness.

  value   proofs/s over K steps with the K witnesses already resident in HBM,
          timed between CUDA events with a barrier and synchronize on both
          sides, max over ranks (N GPUs run N independent replicas: weak).
  e2e     the same through the reference-facing C ABI call with host buffers:
          each step copies its witness from pinned host memory to the device
          and reads the MSM window sums back; p50/p99 per-proof latency too.
  roofline  the dominant kernel (most device time in the timed region), its
          algorithmic work per launch / its average launch duration (CUDA
          events on its own stream) against the measured peak.
  cpu_baseline  the CPU oracle (a C restatement of the reference's CPU
          prover) proving the same circuit on this host's cores.

`--impl reference` times the reference's CPU prover restated in C (the
reference is Rust and cannot be built on this image): the faithful port of its
fast algorithms (oracle/port_*.c), on inputs from the oracle's own generator,
rank 0 only; that arm loads no product code.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
N_CONSTRAINTS = 1_100_000
N_INPUTS, N_PUBLIC = 256, 16
CIRCUIT_SEED, TOXIC_SEED = 21, 0x5EED
FQ_MUL_IMAD = 264            # 8x32-bit CIOS Montgomery product: 32-bit multiply-adds
FQ_SQR_IMAD = 208            # separated squaring: 36 limb products + 8 x 17 for the reduction
FQ2_MUL_IMAD = 3 * 128 + 2 * 136   # three 8x8-limb products, two Montgomery reductions
FQ_MUL_SUB_IMAD = 2 * 128 + 136    # a b - c d: two 8x8-limb products, one reduction
# 32-bit multiply-adds per mixed addition (madd-2008-s, 8M + 2S): G1 squares with
# the separated squaring and forms Y3 = R (Q - X3) - Y1 PPP with one reduction;
# G2 runs all ten as Fq2 products with deferred reduction (656 IMAD each: its two
# squares as products too, which measured faster than separate Fq2 squares)
MADD_IMAD = {"msm_accumulate_g1": 6 * FQ_MUL_IMAD + 2 * FQ_SQR_IMAD + FQ_MUL_SUB_IMAD,
             "msm_accumulate_g2": 10 * FQ2_MUL_IMAD}
MADD_WORK = {"msm_accumulate_g1": "6 Fq products x 264 + 2 Fq squares x 208 + 1 product difference x 392 IMAD",
             "msm_accumulate_g2": "10 Fq2 products x 656 IMAD"}


# g16_ntt modes (CpuNtt, crates/ntt/src/lib.rs:415-584) by bench name
NTT_MODES = {"forward": 0, "inverse": 1, "intt-coset-ntt": 2, "coset": 3}
NTT_WHAT = {"forward": "Fr NTT forward", "inverse": "Fr NTT inverse (with 1/n)",
            "intt-coset-ntt": "Fr iNTT -> coset -> NTT (intt_coset_ntt)",
            "coset": "Fr coset NTT (distribute_powers(shift) then forward)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--constraints", type=int, default=N_CONSTRAINTS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-oracle-check", action="store_true",
                   help="skip comparing a timed proof (and the batched proofs) with the oracle's")
    p.add_argument("--workload", default="prove", choices=["prove", "msm-g1", "msm-g2", "ntt", "batch", "serve"],
                   help="prove (default): full proofs; msm-g1/msm-g2/ntt: the standalone primitives")
    p.add_argument("--log-n", type=int, default=20, help="primitive size 2^log_n")
    p.add_argument("--dist", type=int, default=0, help="MSM scalars: 0 uniform, 1 = 70%% in {0,1}")
    p.add_argument("--ntt-mode", default="intt-coset-ntt", choices=list(NTT_MODES),
                   help="ntt workload: the transform (CpuNtt::ntt forward/inverse, coset, intt_coset_ntt)")
    p.add_argument("--lanes", type=int, default=4, help="served proving: concurrent proofs")
    p.add_argument("--no-autotune", action="store_true", help="batched proving: keep the cost model's tuning")
    p.add_argument("--no-mix", action="store_true",
                   help="prove: skip the batched and served summaries attached to the plain-prove line")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class Ranks:
    """One process per GPU, as torchrun launches them: a barrier and the max over
    ranks through torch.distributed (NCCL between GPUs; gloo where no GPU is
    used).  Proofs are independent, so nothing else crosses ranks: each rank
    proves its own witnesses (witness_seed) on its own replica of the key."""

    def __init__(self, backend="nccl", timeout_s=600):
        import datetime
        import torch
        self.rank, self.local_rank, self.world = dist_env()
        self.dist = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if self.world > 1:
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        if not self.dist:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def witness_seed(rank, step):
    """Distinct witnesses per rank and step."""
    return rank * 1_000_000 + step


def whole_job_rate(world, steps, max_ms):
    """Units all ranks processed over the slowest rank's time (weak scaling)."""
    return world * steps / (max_ms / 1e3)


def workload_name(nc, domain, n_vars):
    return "groth16 prove, synthetic R1CS %d constraints (domain 2^%d, %d wires), BN254" % (
        nc, domain.bit_length() - 1, n_vars)


def fr_mont_bytes(x):
    """A field element of Fr as 32 Montgomery-form bytes."""
    return ((int(x) << 256) % R_MOD).to_bytes(32, "little")


def blinders(i):
    import random
    rng = random.Random(1000 + i)
    return fr_mont_bytes(rng.randrange(1, R_MOD)), fr_mont_bytes(rng.randrange(1, R_MOD))


# The reference's own published CPU prove of this workload's shape, for context
# beside the CPU baseline timed here.
PUBLISHED_CPU = {"ms": 625.7, "proofs_per_s": 1e3 / 625.7,
                 "what": "reference CPU prover (Rust, AVX-512 IFMA field code), warm anon-aadhaar prove: "
                         "1,115,080 constraints, domain 2^21, 16-vCPU c7i.4xlarge",
                 "source": "bench/results/x86-ntt-2026-10-13.md:39"}


def host_cpu():
    """This host's CPU model and logical core count."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        """Start sampling every 50 ms and return once the first sample is in, so the
        samples cover the region timed next."""
        self.first = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        import select
        ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
        if ready:
            self.first = self.proc.stdout.readline()   # taken before the timed region: not counted

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def make_key(sc, toxic, device_ok=True):
    """The synthetic .zkey, its point sections on this rank's GPU when there is one
    (the same bytes as the host generator)."""
    if device_ok:
        try:
            import torch
            if torch.cuda.is_available():
                return sc.zkey(toxic, device=dist_env()[1])
        except ImportError:
            pass
    return sc.zkey(toxic)


def key_cache_path(seed, nc, toxic):
    return os.path.join(os.environ.get("G16_BENCH_CACHE", "/tmp"), "g16b200_bench_%d_%d_%d.zkey" % (seed, nc, toxic))


def cached_key(seed, nc, toxic, make):
    """The workload's .zkey, cached under /tmp so repeated runs on one host skip the key
    generation.  The product's generator and the oracle's give the same bytes for the same
    seeds (tests/test_port.py), so either arm may fill the cache for the other."""
    path = key_cache_path(seed, nc, toxic)
    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError:
        pass
    zk = make()
    try:
        with open(path + ".tmp", "wb") as f:
            f.write(zk)
        os.replace(path + ".tmp", path)
    except OSError:
        pass
    return zk


def synth_key(sc, nc, seed=CIRCUIT_SEED, toxic=TOXIC_SEED, device_ok=True):
    """The workload's .zkey from the product's generator (point sections on this rank's GPU)."""
    return cached_key(seed, nc, toxic, lambda: make_key(sc, toxic, device_ok))


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    return O


def cpu_prove_rate(zk, sc, n_proofs):
    """The oracle proving n_proofs different witnesses of the same circuit, all host threads."""
    O = oracle_module()
    ok = O.Zkey(zk)
    threads = O.max_threads()
    times = []
    for i in range(n_proofs):
        w = sc.witness(10_000 + i)
        r, s = blinders(10_000 + i)
        t0 = time.perf_counter()
        ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        times.append(time.perf_counter() - t0)
    ok.close()
    return times, threads


def oracle_proofs(zk, jobs):
    """The oracle's proofs of [(witness_mont, r_mont, s_mont), ...] on one key, with the
    time each took (all host threads)."""
    O = oracle_module()
    ok = O.Zkey(zk)
    out = []
    for w, r, s in jobs:
        t0 = time.perf_counter()
        p = ok.prove(w, O.from_bytes(r), O.from_bytes(s))
        out.append((p, time.perf_counter() - t0))
    ok.close()
    return out, O.max_threads()


def run_reference(args):
    """The reference's CPU prover (its fast algorithms restated in C: oracle/port_*.c) on the
    same workload, on all host threads, with inputs from the oracle's own generator: this arm
    loads no product code.  Every proof passes the oracle's pairing check, the first equals the
    oracle's plain prover's proof, and one proof is also timed on one core."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    O = oracle_module()
    sc = O.Synth(CIRCUIT_SEED, args.constraints, N_INPUTS, N_PUBLIC)
    zk = cached_key(CIRCUIT_SEED, args.constraints, TOXIC_SEED, lambda: sc.zkey(TOXIC_SEED))
    ok = O.Zkey(zk)
    port = O.PortProver(ok)
    threads = O.max_threads()
    pub = 32 * N_PUBLIC
    times, verified, first = [], 0, None
    for i in range(args.warmup + args.steps):
        seed = witness_seed(0, i)
        w = sc.witness(seed)
        r, s = blinders(seed)
        t0 = time.perf_counter()
        p = port.prove(w, r, s)
        times.append(time.perf_counter() - t0)
        verified += ok.verify(w[32:32 + pub], p)
        if i == args.warmup:
            first = (w, r, s, p)
    w, r, s, p = first
    exact = p == ok.prove(w, O.from_bytes(r), O.from_bytes(s))
    O.set_threads(1)
    t0 = time.perf_counter()
    port.prove(w, r, s)
    one_core = time.perf_counter() - t0
    O.set_threads(threads)
    timed = times[args.warmup:]
    value = len(timed) / sum(timed)
    cpu = dict(host_cpu(), value=value, unit="proofs/s", cores=threads, kind="port",
               sample="%d full proofs of the workload (after %d warm-up) by the reference CPU prover's algorithms "
                      "restated in C (batch-affine MSM fill, five MSMs concurrently, 2^11-blocked intt_coset_ntt), "
                      "OpenMP over all host threads" % (len(timed), args.warmup),
               one_core={"value": 1 / one_core, "unit": "proofs/s", "ms": 1e3 * one_core,
                         "sample": "1 full proof on one thread"})
    line = {
        "impl": "reference", "metric": "proofs/s", "value": value, "unit": "proofs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(timed) / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (BN254 Montgomery, exact)",
        "data": "synthetic",
        "config": {"workload": workload_name(args.constraints, sc.domain_size, sc.n_vars),
                   "n_constraints": args.constraints, "domain": sc.domain_size, "n_vars": sc.n_vars},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1e3 * statistics.median(timed),
        "parity": {"pairing_checked": verified, "of": len(times), "bit_exact_vs_oracle": exact},
        "reference_published_cpu": PUBLISHED_CPU,
        "note": "the reference is Rust (ark-* 0.5 not vendored, no cargo here); this arm times its CPU prover's "
                "algorithms restated in C, the portable path without AVX-512 IFMA",
    }
    port.close()
    ok.close()
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import snarkrs_b200 as S
    ranks = Ranks("nccl")
    rank, local_rank, world = ranks.rank, ranks.local_rank, ranks.world
    barrier, max_over_ranks = ranks.barrier, ranks.max
    torch.cuda.set_device(local_rank)
    backend = S.CudaBackend(local_rank)
    sc = S.SynthCircuit(CIRCUIT_SEED, args.constraints, N_INPUTS, N_PUBLIC)
    zk = synth_key(sc, args.constraints) if rank == 0 or world == 1 else None
    if world > 1:
        barrier()
        zk = synth_key(sc, args.constraints)
    pk = S.ProvingKey.from_bytes(zk, check_points=False)
    t_prep = time.perf_counter()
    circ = backend.prepare(pk)
    t_prep = time.perf_counter() - t_prep
    K, W = args.steps, args.warmup
    nbytes = 32 * sc.n_vars
    # per-step witnesses (different seeds per rank and step), in pinned host memory
    wits = []
    for i in range(W + K):
        t = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = memoryview(sc.witness(witness_seed(rank, i)))
        wits.append(t)
    bl = [blinders(witness_seed(rank, i)) for i in range(W + K)]
    # device-resident copies for the kernel-side number
    dwit = [torch.empty(nbytes, dtype=torch.uint8, device="cuda") for _ in range(W + K)]
    for d, h in zip(dwit, wits):
        d.copy_(h)
    torch.cuda.synchronize()

    # ---- value: inputs resident in HBM ----
    for i in range(W):
        circ.prove_with_blinders_device(dwit[i].data_ptr(), sc.n_vars, *bl[i])
    clocks = Clocks(local_rank)
    barrier()
    torch.cuda.synchronize()
    launches0 = S.launch_count()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    proofs = []
    e0.record()
    for i in range(W, W + K):
        proofs.append(circ.prove_with_blinders_device(dwit[i].data_ptr(), sc.n_vars, *bl[i]))
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    launches = int(S.launch_count() - launches0)
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = whole_job_rate(world, K, ms)

    # ---- e2e: host buffers through the C ABI, pinned witness copied every step ----
    lat = []
    e2e_proofs = []
    barrier()
    torch.cuda.synchronize()
    t_all = time.perf_counter()
    for i in range(W, W + K):
        t0 = time.perf_counter()
        e2e_proofs.append(circ.prove_with_blinders(wits[i].numpy(), *bl[i]))
        lat.append(time.perf_counter() - t0)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t_all)
    e2e_value = whole_job_rate(world, K, 1e3 * e2e_s)
    readback = int(circ.readback_bytes())

    # ---- parity of the timed proofs (after timing): each passes the product's pairing
    # check, the e2e proofs equal the device-resident ones, and (rank 0, below) the first
    # timed proof equals the oracle's proof of the same witness with the same r and s ----
    pub_bytes = 32 * N_PUBLIC
    for i, p in zip(range(W, W + K), proofs):
        circ.verify(bytes(wits[i].numpy()[32:32 + pub_bytes]), p)      # raises VerifyError
    same_e2e = all(a == b for a, b in zip(proofs, e2e_proofs))

    # ---- per-kernel times: the same proofs replayed with every stage on one stream ----
    # (the timed region overlaps three streams, so event spans there would include
    # concurrent kernels; the serialized replay gives each kernel's own duration)
    circ.set_serial(True)
    S.kernel_timing_reset()
    S.kernel_timing(True)
    for i in range(W, W + K):
        circ.prove_with_blinders_device(dwit[i].data_ptr(), sc.n_vars, *bl[i])
    S.kernel_timing(False)
    kern = S.kernel_timing_report()
    kbytes = S.kernel_timing_bytes()
    circ.set_serial(False)

    if rank != 0:
        ranks.close()
        return

    # ---- roofline of the dominant kernel ----
    peaks, peak_kind = measured_peaks()
    imad_peak = S.imad_peak(backend)
    dom = max(kern.items(), key=lambda kv: kv[1][0])
    name, (tot_ms, n_launch, units) = dom[0], dom[1]
    roof = {"kernel": name, "launches": n_launch, "avg_ms": tot_ms / max(n_launch, 1),
            "measured_over": "serialized replay of the %d timed proofs (CUDA events per launch)" % K}
    if name in MADD_IMAD:
        imad_per_launch = units / max(n_launch, 1) * MADD_IMAD[name]
        achieved = imad_per_launch / (roof["avg_ms"] / 1e3)
        roof.update({"bound": "imad", "achieved": achieved / 1e12, "peak": imad_peak / 1e12, "unit": "TIMAD/s",
                     "frac": achieved / imad_peak, "peak_source": "measured in this run by the mad.lo/mad.hi "
                                                                    "issue-rate probe (g16_imad_peak)",
                     "work_per_launch": "%.0f mixed additions x (%s)" % (
                         units / max(n_launch, 1), MADD_WORK[name])})
    roof["traffic"] = traffic_for("prove-%d" % args.constraints, name)
    # whole-proof integer work: MSM mixed additions (measured counters) + the NTT chain
    n_dom = sc.domain_size
    log_n = n_dom.bit_length() - 1
    ntt_muls = 6 * (n_dom // 2) * log_n + 3 * n_dom + 2 * n_dom
    msm_imad = sum(kern.get(k, (0, 0, 0))[2] * MADD_IMAD[k] for k in MADD_IMAD) / K
    proof_imad = msm_imad + ntt_muls * FQ_MUL_IMAD
    whole = {"imad_per_proof": proof_imad, "achieved_timad_s": proof_imad / (ms / K / 1e3) / 1e12,
             "frac_of_peak": proof_imad / (ms / K / 1e3) / imad_peak,
             "note": "algorithmic IMAD of a whole proof / timed ms per proof, against the measured IMAD peak"}
    share = {k: round(v[0] / sum(x[0] for x in kern.values()), 4) for k, v in kern.items()}
    per_kernel = kernel_rooflines(kern, kbytes, imad_peak, peaks["hbm_gbs"])
    t = circ.stage_timings()

    cpu = None
    parity = {"pairing_checked": K, "e2e_equals_device_resident": same_e2e}
    if not args.no_oracle_check:
        # the oracle proves the first timed witness with its r and s
        (want, dt), = oracle_proofs(zk, [(bytes(wits[W].numpy()), bl[W][0], bl[W][1])])[0]
        parity["bit_exact_vs_oracle"] = proofs[0].to_bytes() == want
        parity["oracle_checked"] = "step %d of %d (witness seed %d)" % (W, W + K, witness_seed(rank, W))
    if not args.no_cpu_baseline and world == 1:
        # the reference CPU prover's algorithms (oracle/port_*.c) prove the same witness
        O = oracle_module()
        ok = O.Zkey(zk)
        port = O.PortProver(ok)
        w0 = bytes(wits[W].numpy())
        t0 = time.perf_counter()
        got = port.prove(w0, *bl[W])
        dt = time.perf_counter() - t0
        parity["cpu_baseline_proof_equal"] = got == proofs[0].to_bytes()
        cpu = dict(host_cpu(), value=1 / dt, unit="proofs/s", cores=O.max_threads(), kind="port",
                   sample="1 full proof of the same workload (the first timed witness) by the reference CPU "
                          "prover's algorithms restated in C (batch-affine MSM fill, five MSMs concurrently, "
                          "2^11-blocked intt_coset_ntt; OpenMP, all host threads), %.2f s" % dt,
                   reference_published=PUBLISHED_CPU)
        port.close()
        ok.close()
    line = {
        "metric": "proofs/s", "value": value, "unit": "proofs/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (BN254 Fq/Fr Montgomery limbs, exact)", "data": "synthetic",
        "config": {"workload": workload_name(args.constraints, sc.domain_size, sc.n_vars),
                   "n_constraints": args.constraints, "domain": sc.domain_size, "n_vars": sc.n_vars,
                   "l2": "no flush: the resident key (%.0f MB) and per-step witnesses exceed the 126 MB L2" %
                         (circ.device_bytes() / 1e6),
                   "replicas": world,
                   "prepare_s": round(t_prep, 3)},
        "e2e": {"value": e2e_value, "unit": "proofs/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": readback, "p50_ms": 1e3 * statistics.median(lat),
                "p99_ms": 1e3 * sorted(lat)[min(len(lat) - 1, int(0.99 * len(lat)))]},
        "roofline": roof,
        "whole_proof_roofline": whole,
        "kernel_share": share,
        "kernel_ms_per_step": {k: round(v[0] / K, 4) for k, v in kern.items()},
        "kernel_launches_per_step": {k: v[1] / K for k, v in kern.items()},
        "kernel_rooflines": per_kernel,
        "stage_us_total": t,
        "gpu_launches": launches,
        "parity": parity,
        "bit_exact_vs_oracle": parity.get("bit_exact_vs_oracle"),
        "clocks": clk,
        "hbm_peak_gbs": peaks.get("hbm_gbs"), "hbm_peak_source": peak_kind,
        "reference_published": "T4 warm CUDA prove at domain 2^21: 1263 ms (bench/results/cuda-size-sweep-2026-11-10.md:26)",
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if world == 1 and not args.no_mix:
        circ.close()
        # the metric's other half: batched and served proving against plain one-at-a-time
        try:
            b = run_batch(args, backend, emit=False, steps=min(args.steps, 3))
            line["batched"] = {"workload": b["config"]["workload"], "value": b["value"], "unit": "proofs/s",
                               "plain_value": b["plain"]["value"], "plain_p50_ms": b["plain"]["p50_ms"],
                               "plain_p99_ms": b["plain"]["p99_ms"], "speedup_vs_plain": b["speedup_vs_plain"],
                               "bit_exact_vs_plain": b["bit_exact_vs_plain"],
                               "bit_exact_vs_oracle": b["bit_exact_vs_oracle"],
                               "p50_ms": b["p50_ms"], "p99_ms": b["p99_ms"],
                               "plain_queued_p50_ms": b["plain"]["queued_p50_ms"],
                               "plain_queued_p99_ms": b["plain"]["queued_p99_ms"],
                               "kernel_launches_per_batch": b["kernel_launches_per_batch"],
                               "per_instance_tuning": b["config"]["per_instance_tuning"]}
        except Exception as e:   # the plain-prove line above stands on its own
            line["batched"] = {"error": repr(e)[:300]}
        try:
            v = run_serve(args, backend, emit=False, fracs=(1.5,), n_req=300)
            top = v["sweep"][-1]
            line["served"] = {"workload": v["config"]["workload"], "offered_fraction_of_plain_capacity": 1.5,
                              "requests": top["served"]["requests"],
                              "value": top["served"]["throughput"], "unit": "proofs/s",
                              "p50_ms": top["served"]["p50_ms"], "p99_ms": top["served"]["p99_ms"],
                              "plain_fifo": {k: top["plain_fifo"][k] for k in ("throughput", "p50_ms", "p99_ms")},
                              "stats": top["served"]["stats"],
                              "results_identical_alone_and_in_mix": v["results_identical_alone_and_in_mix"]}
        except Exception as e:
            line["served"] = {"error": repr(e)[:300]}
    print(json.dumps(line), flush=True)
    ranks.close()


def traffic_for(workload, name):
    """DRAM bytes per launch from the committed ncu summary for this workload and kernel, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            entry = json.load(f).get(workload, {}).get(name)
    except (OSError, ValueError, AttributeError):
        return None
    return entry.get("bytes_per_launch") if isinstance(entry, dict) else None


NTT_KERNELS = ("ntt_pass_dif", "ntt_pass_dit", "ntt_mid_fused")


def kernel_rooflines(kern, kbytes, imad_peak, hbm_peak):
    """Per kernel class: integer-multiply rate (MSM accumulate: mixed additions;
    NTT passes: Fr products) and HBM rate (NTT passes, MSM sort) against the
    measured peaks, averaged over its launches."""
    out = {}
    for name, (ms, launches, units) in kern.items():
        if ms <= 0:
            continue
        row = {}
        imad = None
        if name in MADD_IMAD:
            imad = units * MADD_IMAD[name]
        elif name in NTT_KERNELS:
            imad = units * FQ_MUL_IMAD
        if imad:
            rate = imad / (ms / 1e3)
            row.update({"timad_s": rate / 1e12, "imad_frac": rate / imad_peak})
        if name in kbytes:
            gbs = kbytes[name] / (ms / 1e3) / 1e9
            row.update({"hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak})
        if row:
            row["launches"] = launches
            out[name] = row
    return out


def reference_window_size(m):
    """c of the reference CPU MSM for m general scalars (crates/msm/src/lib.rs:160-172): the c in
    3..16 minimising ceil(255/c) * (m + 3 * 2^(c-1))."""
    best, best_cost = 3, None
    for c in range(3, 17):
        cost = -(-255 // c) * (m + 3 * (1 << (c - 1)))
        if best_cost is None or cost < best_cost:
            best, best_cost = c, cost
    return best


def msm_work_model(scalars, g2):
    """Algorithmic work of one MSM by the reference's model: m general (not 0 or 1) scalars,
    c = window_size(m), W = ceil(255/c), B = 2^(c-1); Fq products = 10 m W + 28 B W plus 10 per
    scalar equal to 1, three times that in G2; 264 IMAD per Fq product."""
    import numpy as np
    v = np.frombuffer(scalars, dtype=np.uint64).reshape(-1, 4)
    high_zero = (v[:, 1] | v[:, 2] | v[:, 3]) == 0
    zeros = int(np.count_nonzero(high_zero & (v[:, 0] == 0)))
    ones = int(np.count_nonzero(high_zero & (v[:, 0] == 1)))
    m = len(v) - zeros - ones
    c = reference_window_size(m) if m else 3
    w, b = -(-255 // c), 1 << (c - 1)
    muls = (10 * m * w + 28 * b * w + 10 * ones) * (3 if g2 else 1)
    return {"general_scalars": m, "ones": ones, "zeros": zeros, "c": c, "fq_products": muls,
            "imad": muls * FQ_MUL_IMAD}


def run_primitive(args):
    """Standalone MSM (points/s) or NTT (elements/s) on device-resident inputs."""
    import torch
    import snarkrs_b200 as S
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    backend = S.CudaBackend(local_rank)
    n = 1 << args.log_n
    K, W = args.steps, args.warmup
    g2 = args.workload == "msm-g2"
    if args.workload.startswith("msm"):
        bases = S.synth_points(2 if g2 else 1, 77 + rank, n)
        scal = S.synth_scalars(78 + rank, n, args.dist)
        d_b = torch.frombuffer(bytearray(bases), dtype=torch.uint8).cuda()
        d_s = torch.frombuffer(bytearray(scal), dtype=torch.uint8).cuda()
        msm = S.CudaMsm(backend)
        fn = msm.msm_g2_device if g2 else msm.msm_g1_device
        step = lambda: fn(d_b.data_ptr(), d_s.data_ptr(), n)
        unit, what = "points/s", "%s MSM, N = 2^%d, %s scalars" % (
            "G2" if g2 else "G1", args.log_n, "70% {0,1}" if args.dist else "uniform")
        host = lambda: (msm.msm_g2 if g2 else msm.msm_g1)(bases, scal)
        h2d = len(bases) + len(scal)
    else:
        data = S.synth_scalars(79 + rank, n, 0)
        d = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
        ntt = S.CudaNtt(backend)
        mode = NTT_MODES[args.ntt_mode]
        step = lambda: ntt.ntt_device(mode, args.log_n, d.data_ptr())
        unit, what = "elements/s", "%s, n = 2^%d" % (NTT_WHAT[args.ntt_mode], args.log_n)
        host = {"forward": lambda: ntt.ntt(data), "inverse": lambda: ntt.ntt(data, inverse=True),
                "coset": lambda: ntt.coset_ntt(data), "intt-coset-ntt": lambda: ntt.intt_coset_ntt(data)}[args.ntt_mode]
        h2d = len(data)
    for _ in range(W):
        step()
    S.kernel_timing_reset()
    S.kernel_timing(True)
    torch.cuda.synchronize()
    l0 = S.launch_count()
    clocks = Clocks(local_rank)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(K):
        step()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    S.kernel_timing(False)
    kern = S.kernel_timing_report()
    ms = e0.elapsed_time(e1)
    t0 = time.perf_counter()
    for _ in range(K):
        host()
    e2e_s = time.perf_counter() - t0
    line = {"metric": unit, "value": n * K / (ms / 1e3), "unit": unit, "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 (BN254 Montgomery limbs, exact)", "data": "synthetic", "config": {"workload": what},
            "e2e": {"value": n * K / e2e_s, "unit": unit, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": (128 if g2 else 64) if args.workload.startswith("msm") else h2d},
            "gpu_launches": int(S.launch_count() - l0), "clocks": clk,
            "kernel_share": {k: round(v[0] / sum(x[0] for x in kern.values()), 4) for k, v in kern.items()}}
    kbytes = S.kernel_timing_bytes()
    peaks, peak_kind = measured_peaks()
    imad_pk = S.imad_peak(backend)
    per_kernel = kernel_rooflines(kern, kbytes, imad_pk, peaks["hbm_gbs"])
    dom = max(kern.items(), key=lambda kv: kv[1][0])
    name, (tot_ms, n_launch, units) = dom[0], dom[1]
    roof = {"kernel": name, "launches": n_launch, "avg_ms": tot_ms / max(n_launch, 1)}
    r = per_kernel.get(name, {})
    if r.get("imad_frac", 0) >= r.get("hbm_frac", 0) and "imad_frac" in r:
        roof.update({"bound": "imad", "achieved": r["timad_s"], "peak": imad_pk / 1e12, "unit": "TIMAD/s",
                     "frac": r["imad_frac"], "peak_source": "measured in this run (g16_imad_peak)"})
    elif "hbm_frac" in r:
        roof.update({"bound": "hbm", "achieved": r["hbm_gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": r["hbm_frac"], "peak_source": peak_kind})
    roof["traffic"] = traffic_for("%s-2^%d" % (args.workload, args.log_n), name)
    line["roofline"] = roof
    line["kernel_rooflines"] = per_kernel
    if args.workload.startswith("msm"):
        # the whole MSM against the reference's work model (its window size, 10 products per
        # bucket addition, 28 B W for the bucket reduction), per timed step
        wm = msm_work_model(scal, g2)
        rate = wm["imad"] / (ms / K / 1e3)
        wm.update({"achieved": rate / 1e12, "peak": imad_pk / 1e12, "unit": "TIMAD/s", "frac": rate / imad_pk,
                   "note": "reference work model (crates/msm/src/lib.rs:160-172) / timed ms per MSM"})
        line["work_model_roofline"] = wm
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        O.build()
        t0 = time.perf_counter()
        if args.workload.startswith("msm"):
            (O.msm_g2 if g2 else O.msm_g1)(bases, scal)
        else:
            O.ntt(args.log_n, NTT_MODES[args.ntt_mode], data)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n / dt, "unit": unit, "cores": O.max_threads(), "kind": "port",
                                "sample": "1 run of the same input on the C restatement, %.2f s" % dt}
    print(json.dumps(line), flush=True)


BATCH_LANES = 8   # g16_prove_batch's default lane count (G16_BATCH_LANES)


def batch_circuits(seed=3, count=8, lo=12, hi=18):
    """The batched workload's circuits: sizes log-uniform over 2^lo..2^hi constraints, seeded."""
    import random
    rng = random.Random(seed)
    return sorted(int(2 ** rng.uniform(lo, hi)) for _ in range(count))


def run_batch(args, backend=None, emit=True, steps=None):
    """64 proofs over 8 circuits of uneven size: one batched submission vs one at a time."""
    import snarkrs_b200 as S
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    backend = backend or S.CudaBackend(local_rank)
    sizes = batch_circuits()
    circs, wits, tunes, zks = [], [], [], []
    t_tune = 0.0
    for i, nc in enumerate(sizes):
        sc = S.SynthCircuit(500 + i, nc, N_INPUTS, N_PUBLIC)
        zks.append(make_key(sc, TOXIC_SEED + i))
        circs.append(backend.prepare(S.ProvingKey.from_bytes(zks[-1], check_points=False)))
        wits.append([sc.witness(1000 * i + j) for j in range(8)])
        if not args.no_autotune:
            # the batched objective: as many proofs in flight as prove_batch has lanes
            t0 = time.perf_counter()
            tunes.append(dict(circs[-1].autotune(wits[-1][0], concurrency=BATCH_LANES), constraints=nc))
            t_tune += time.perf_counter() - t0
        else:
            tunes.append(dict(circs[-1].tuning(), constraints=nc))
    jobs, job_circuit = [], []
    for j in range(8):
        for i in range(len(sizes)):
            r, s_ = blinders(100 * i + j)
            jobs.append((circs[i], wits[i][j], r, s_))
            job_circuit.append(i)
    # warm-up: every circuit once on its own, then one batch (workspaces, graphs)
    for c, w, r, s_ in jobs[:len(sizes)]:
        c.prove_with_blinders(w, r, s_)
    backend.prove_batch(jobs)
    lat, plain = [], []
    t0 = time.perf_counter()
    for c, w, r, s_ in jobs:
        t1 = time.perf_counter()
        plain.append(c.prove_with_blinders(w, r, s_))
        lat.append(time.perf_counter() - t1)
    t_plain = time.perf_counter() - t0
    best, out, done = None, None, None
    steps = steps or args.steps
    for _ in range(max(1, steps)):
        d = []
        t0 = time.perf_counter()
        out = backend.prove_batch(jobs, done_ms=d)
        dt = time.perf_counter() - t0
        if best is None or dt < best:
            best, done = dt, d
    assert all(a == b for a, b in zip(out, plain)), "batched proofs differ from single proofs"
    # latency of a batch submitted at once: each proof's completion time from the
    # submission, batched, against the same 64 jobs queued FIFO one at a time
    fifo, acc = [], 0.0
    for x in lat:
        acc += x
        fifo.append(1e3 * acc)
    done, fifo = sorted(done), sorted(fifo)
    pct = lambda v, q: v[min(len(v) - 1, int(q * len(v)))]
    # one more submission with kernel timing on (stage by stage, no graph): each kernel
    # class's launches and device time for the whole batch
    S.kernel_timing_reset()
    S.kernel_timing(True)
    backend.prove_batch(jobs)
    S.kernel_timing(False)
    kern = S.kernel_timing_report()
    exact = None
    if not args.no_oracle_check:
        exact = True
        for i in range(len(sizes)):
            mine = [(k, jobs[k]) for k in range(len(jobs)) if job_circuit[k] == i]
            want, _ = oracle_proofs(zks[i], [(w, r, s_) for _, (_, w, r, s_) in mine])
            exact &= all(out[k].to_bytes() == p for (k, _), (p, _) in zip(mine, want))
    lat.sort()
    line = {"metric": "proofs/s", "value": len(jobs) / best, "unit": "proofs/s", "n_gpus": 1, "steps": steps,
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 (BN254 Montgomery limbs, exact)", "data": "synthetic",
            "config": {"workload": "batched prove: 64 proofs over 8 synthetic circuits, sizes log-uniform "
                                   "over 2^12..2^18 constraints, 8 witnesses each",
                       "constraints": sizes,
                       "per_instance_tuning": "autotuner (g16_autotune, %d proofs in flight, %.1f s for 8 "
                                              "circuits)" % (BATCH_LANES, t_tune)
                       if not args.no_autotune else "cost model", "tuning": tunes},
            "plain": {"value": len(jobs) / t_plain, "unit": "proofs/s", "p50_ms": 1e3 * lat[len(lat) // 2],
                      "p99_ms": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                      "queued_p50_ms": pct(fifo, 0.5), "queued_p99_ms": pct(fifo, 0.99)},
            "p50_ms": pct(done, 0.5), "p99_ms": pct(done, 0.99),
            "latency_note": "p50/p99: completion time of each proof from the submission of all 64 at once; "
                            "plain.queued_*: the same 64 queued FIFO one at a time; plain.p50/p99: one proof alone",
            "kernel_launches_per_batch": {k: v[1] for k, v in kern.items()},
            "kernel_ms_per_batch": {k: round(v[0], 4) for k, v in kern.items()},
            "batch_ms": 1e3 * best, "speedup_vs_plain": t_plain / best,
            "bit_exact_vs_plain": True, "bit_exact_vs_oracle": exact}
    for c in circs:
        c.close()
    if emit:
        print(json.dumps(line), flush=True)
    return line


# Circuits labelled 2^k constraints have domain 2^k and about 0.52 * 2^k active
# rows, the convention of the 2^21-constraint prove (1.1M rows, domain 2^21);
# the largest one is that very circuit.
SERVE_LOGS = [14, 16, 17, 18, 20, 21]
SERVE_WEIGHTS = [30, 25, 20, 12, 8, 5]


def serve_circuits():
    out = []
    for k in SERVE_LOGS:
        if k == 21:
            out.append((CIRCUIT_SEED, N_CONSTRAINTS))
        else:
            out.append((700 + k, (N_CONSTRAINTS << k) >> 21))
    return out


def run_serve(args, backend=None, emit=True, fracs=(0.5, 0.9, 1.5), n_req=None):
    """Poisson arrivals over six circuits; continuous batching vs plain FIFO, p50/p99."""
    import random
    import statistics as st
    import snarkrs_b200 as S
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    backend = backend or S.CudaBackend(local_rank)
    keys, wits = [], []
    for seed, nc in serve_circuits():
        sc = S.SynthCircuit(seed, nc, N_INPUTS, N_PUBLIC)
        keys.append(synth_key(sc, nc, seed))
        wits.append([sc.witness(7000 + 10 * len(wits) + j) for j in range(2)])
    budget = 120 << 30

    def arrivals(rate, n_req, seed):
        rng = random.Random(seed)
        reqs, t = [], 0.0
        for j in range(n_req):
            t += rng.expovariate(rate)
            i = rng.choices(range(len(keys)), weights=SERVE_WEIGHTS)[0]
            reqs.append((t, i, j))
        return reqs

    def play(srv, reqs, blind_base):
        tickets = []
        t0 = time.perf_counter()
        for (ta, i, j) in reqs:
            delay = t0 + ta - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            r, s_ = blinders(blind_base + j)
            tickets.append((srv.submit(i, wits[i][j % 2], r, s_), i, j))
        return t0, tickets

    def run(lanes, rate, n_req, seed, max_batch=64):
        srv = S.ProofServer(backend, budget, lanes, max_batch)
        for i, k in enumerate(keys):
            srv.register_key(i, k)
        # warm the server outside the measurement with the same arrival process
        # (other draws): keys prepared, as many workspaces and engines as the load
        # keeps busy, their buffers at size and CUDA graphs captured, as in a
        # server that has been running
        for i in range(len(keys)):
            r, s_ = blinders(i)
            srv.wait(srv.submit(i, wits[i][0], r, s_))
        _, warm = play(srv, arrivals(rate, n_req, seed + 1000), 20_000)
        for tk, _, _ in warm:
            srv.wait(tk)
        reqs = arrivals(rate, n_req, seed)
        tickets = []
        bs0, allocs0, ss0 = backend.batch_stats(), S.device_alloc_count(), srv.stats()
        t0, tickets = play(srv, reqs, 10_000)
        lat, proofs = [], {}
        for tk, i, j in tickets:
            p, q, l = srv.wait(tk)
            lat.append(l)
            proofs[j] = p
        t_end = time.perf_counter()
        stats = srv.stats()
        for key in ("batches", "batched", "alone", "submitted", "completed"):   # the timed pass alone
            stats[key] -= ss0[key]
        bs1 = backend.batch_stats()
        stats["engine"] = {k: bs1[k] - bs0[k] for k in bs1}
        stats["device_allocs_in_timed_region"] = S.device_alloc_count() - allocs0
        srv.close()
        lat.sort()
        return {"lanes": lanes, "offered_rate": rate, "requests": n_req,
                "throughput": n_req / (t_end - t0), "p50_ms": lat[len(lat) // 2],
                "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))], "mean_ms": st.mean(lat),
                "stats": stats}, proofs

    # plain capacity: mean service time over the mix, one request at a time
    calib, _ = run(1, 1e6, 60, 1, max_batch=1)     # back-to-back arrivals = saturated FIFO
    cap = calib["throughput"]
    n_req = n_req or max(300, args.steps * 100)
    results = []
    mix_ok = True
    for frac in fracs:
        rate = frac * cap
        plain, pp = run(1, rate, n_req, 42 + int(frac * 10), max_batch=1)
        served, sp = run(args.lanes, rate, n_req, 42 + int(frac * 10))
        mix_ok &= all(pp[j] == sp[j] for j in pp)
        results.append({"offered_fraction_of_plain_capacity": frac, "plain_fifo": plain, "served": served})
    top = results[-1]["served"]
    line = {"metric": "proofs/s", "value": top["throughput"], "unit": "proofs/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 2, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32 (BN254 Montgomery limbs, exact)", "data": "synthetic",
            "config": {"workload": "served prove: Poisson arrivals over 6 synthetic circuits of 2^14, 2^16, 2^17, "
                                   "2^18, 2^20, 2^21 constraints, mix 30/25/20/12/8/5%, 120 GB key budget",
                       "active_rows": [nc for _, nc in serve_circuits()], "lanes": args.lanes,
                       "plain_capacity_proofs_s": cap},
            "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
            "sweep": results, "results_identical_alone_and_in_mix": mix_ok}
    if emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    args = parse()
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "prove":
        run_primitive(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
