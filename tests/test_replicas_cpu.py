"""The multi-GPU form of the bench is replicas: every rank matches its own
frame, and the only cross-rank steps are the timing barrier and the max of the
per-rank times.  Those steps run here on CPU ranks over gloo (world size 2),
with the same functions bench.py calls on NCCL."""
import importlib.util
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = _bench()
        local_ms = [1500.0, 1750.0][rank]
        job_ms = b.job_time(local_ms, world, "cpu")
        dist.barrier()
        e2e = b.job_time([3.0, 2.5][rank], world, "cpu")
        # the reference arm runs on rank 0 only; the others return at once
        ref = b.run_reference(None, rank, world) if rank != 0 else "rank0"
        q.put((rank, job_ms, e2e, b.replica_throughput(4, world, job_ms / 1e3), ref))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, job_ms, e2e, fps, ref in got:
        assert job_ms == 1750.0 and e2e == 3.0
        assert fps == pytest.approx(2 * 4 / 1.75)
    assert got[1][4] is None                     # rank 1 of the reference arm does no work


def test_single_rank_needs_no_process_group():
    b = _bench()
    assert b.job_time(12.5, 1, "cpu") == 12.5
    assert b.replica_throughput(3, 1, 1.5) == 2.0
