"""Replica runs of bench.py (--gpus N under torchrun): every rank runs its own simulation, the
timed region is aggregated as the slowest rank's time, and the whole-job rate counts the slices
of all ranks. Checked with two gloo ranks on the CPU (the aggregation is host logic; the GPU runs
here have one GPU)."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    def reduce_max(x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the device-timed region: rank 1 is the slower one; the end-to-end region: rank 0 is
    value = bench.job_rate(1.0 + rank, 256 * 5, world, reduce_max)
    e2e = bench.job_rate(2.0 - 0.5 * rank, 256 * 5, world, reduce_max)
    q.put((rank, value, e2e))
    dist.destroy_process_group()


def test_job_rate_is_all_slices_over_the_slowest_rank():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r for r, _, _ in out) == [0, 1]
    for _, (value, secs), (e2e, e2e_secs) in out:
        assert secs == 2.0 and value == 2 * 1280 / 2.0
        assert e2e_secs == 2.0 and e2e == 2 * 1280 / 2.0


def test_single_rank_rate_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(0.5, 1280, 1, lambda x: x) == (2560.0, 0.5)


def test_reference_arm_runs_on_rank_0_only(monkeypatch, capsys):
    """Under torchrun the reference arm is timed by rank 0 alone; the other ranks exit at once."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(config="blowout_255", steps=1, warmup=0, cpu_sample_slices=0)
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
