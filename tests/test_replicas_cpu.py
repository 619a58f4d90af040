"""The multi-GPU form of the benchmark on CPU: independent replicas, one per
rank, joined only by the max-over-ranks of the step time (no data-path
collective). Two gloo ranks stand in for two GPUs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, step_ms, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        t = bench.max_over_ranks(step_ms[rank], dist)
        value = bench.replica_throughput(world, 3.288e11, t)
        out.put((rank, t, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    step_ms = [120.0, 131.5]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, step_ms, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(out.get(timeout=5) for _ in range(2))
    for rank, t, value in res:
        assert t == 131.5  # every rank sees the slowest replica's time
        assert value == pytest.approx(2 * 3.288e11 / 0.1315 / 1e9)


def test_single_process_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.0) == 7.0
    assert bench.replica_throughput(1, 1e9, 1000.0) == pytest.approx(1.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.parse_args(["--impl", "reference", "--gpus", "2"])
    bench.run_reference(args)  # returns at once: only rank 0 measures and prints
    assert capsys.readouterr().out == ""
