"""The N > 1 plumbing of bench.py, as torchrun runs it with one process per GPU,
exercised here as two gloo ranks on the CPU: the barrier, the max over ranks that
times a multi-GPU step, distinct witnesses per rank, and the whole-job rate.
Proofs are independent, so these are the only cross-rank operations (replicas)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world)})
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo", timeout_s=60)
    ranks.barrier()
    slowest = ranks.max(100.0 + 25.0 * rank)        # this rank's step time, ms
    seeds = [bench.witness_seed(ranks.rank, i) for i in range(3)]
    rate = bench.whole_job_rate(ranks.world, 10, slowest)
    ranks.close()
    out.put((rank, ranks.world, slowest, seeds, rate))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [2, 2]
    assert [r[2] for r in results] == [125.0, 125.0]            # both ranks see the slowest time
    assert set(results[0][3]).isdisjoint(results[1][3])          # distinct witnesses per rank
    assert results[0][4] == results[1][4] == pytest.approx(2 * 10 / 0.125)


def test_single_process_needs_no_process_group(monkeypatch):
    import sys
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo")
    assert ranks.world == 1 and ranks.max(3.5) == 3.5
    ranks.barrier()
    ranks.close()
