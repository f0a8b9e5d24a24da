"""The multi-GPU plumbing of bench.py on the host: two gloo ranks on 127.0.0.1.

The closest-hit workload runs as independent replicas, one per GPU (each rank walks its own
batch; nothing crosses between ranks on the data path), so what a multi-rank run adds is the
barrier around the timed region, the maximum of the ranks' times and the whole-job rate built
from it, and the reference arm running on rank 0 alone.  These run here without a GPU."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path
from types import SimpleNamespace

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    ranks = bench.Ranks("gloo", timeout_s=60)
    ranks.barrier()
    slowest = ranks.max(0.5 + 0.25 * rank)        # rank r "took" 0.5 + 0.25 r seconds
    rate = bench.whole_job_rate(ranks.world, 1000, 4, slowest)
    ranks.barrier()
    ranks.close()
    out.put((rank, ranks.world, slowest, rate))


def test_two_ranks_agree_on_the_slowest_time_and_the_whole_job_rate():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in results] == [0, 1]
    for _, world, slowest, rate in results:
        assert world == 2
        assert slowest == 0.75                   # the max over ranks, on every rank
        assert rate == 2 * 1000 * 4 / 0.75       # all ranks' units over the slowest rank's time


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, str(ROOT))
    import bench
    ranks = bench.Ranks("gloo")
    assert (ranks.world, ranks.rank) == (1, 0)
    ranks.barrier()
    assert ranks.max(3.5) == 3.5
    ranks.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the reference arm's other ranks exit without work or output."""
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.run_reference(SimpleNamespace(gpus=2, steps=1, warmup=0)) is None
    assert capsys.readouterr().out == ""
