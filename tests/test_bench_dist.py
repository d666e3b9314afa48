"""bench.py's multi-process plumbing on the CPU: two gloo ranks on
127.0.0.1, as torchrun would start them.  The job's time is the slowest
rank's (max over ranks), the job's rate counts every rank's replica, the
launch check rejects a world size that does not match --gpus, and the
reference arm does its work on rank 0 only."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    w, r, local = bench.dist_setup(world)
    dist.init_process_group("gloo", rank=r, world_size=w)
    t = bench.max_over_ranks(1.0 + 0.5 * r, w, "cpu")
    v = bench.aggregate_mlups(1_000_000, 10, t, w)

    class A:
        steps, warmup = 1, 0
    skipped = bench.run_reference_arm(A, w, r) if r != 0 else None
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, t, v, skipped))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, t, v, skipped in res:
        assert t == 1.5  # the slower rank's time on every rank
        assert v == pytest.approx(2 * 1_000_000 * 10 / 1.5 / 1e6)
    assert res[1][3] == 0  # rank 1 of the reference arm exits without work


def test_world_size_must_match(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(SystemExit):
        bench.dist_setup(1)
    monkeypatch.setenv("WORLD_SIZE", "1")
    assert bench.dist_setup(1)[0] == 1
