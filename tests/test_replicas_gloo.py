"""Replica plumbing at world_size 2 over gloo on the host (no GPU).

The multi-GPU path is N independent replicas: this checks the pieces the
benchmark and the batch driver use around them -- barrier, max of device
times, sum of units, whole-job throughput and the split of independent
instances across ranks -- with two real processes.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from tycho2_b200.replicas import ReplicaGroup
    g = ReplicaGroup(backend="gloo", timeout_s=60)
    try:
        g.barrier()
        seconds = 1.0 + rank          # rank 1 is the slow one
        units = 100.0 * (rank + 1)    # ranks may hold different work
        res = {"max": g.max(seconds), "sum": g.sum(units), "rate": g.throughput(units, seconds),
               "shard": g.shard(7), "world": g.world, "device": g.device}
        g.barrier()
        out.put((rank, res))
    finally:
        g.close()


@pytest.mark.timeout(120)
def test_two_gloo_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for r in range(world):
        assert got[r]["world"] == 2 and got[r]["device"] == r
        assert got[r]["max"] == 2.0
        assert got[r]["sum"] == 300.0
        assert got[r]["rate"] == 150.0
    assert got[0]["shard"] == [0, 2, 4, 6] and got[1]["shard"] == [1, 3, 5]


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from tycho2_b200.replicas import ReplicaGroup
    g = ReplicaGroup(backend="gloo")
    assert (g.world, g.rank, g.device) == (1, 0, 0)
    assert g.max(3.5) == 3.5 and g.sum(2) == 2.0 and g.shard(3) == [0, 1, 2]
    assert g.throughput(10, 2) == 5.0
    g.close()
