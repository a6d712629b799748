"""Multi-process replica logic on CPU (gloo, world size 2): source sharding,
max-over-ranks time and whole-job totals, as bench.py uses them on GPUs."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from sygraph_b200 import replicas
        srcs = np.arange(100, 100 + 64 * world, dtype=np.uint32)
        mine = replicas.shard(srcs, rank, world, per_rank=64)
        t = 1.0 + rank  # rank 1 is slower
        edges = 1000.0 * (rank + 1)
        res = {
            "rank": rank,
            "first": int(mine[0]),
            "n": int(mine.size),
            "tmax": replicas.max_over_ranks(t),
            "esum": replicas.sum_over_ranks(edges),
            "rate": replicas.whole_job_rate(edges, t),
        }
        q.put(res)
    finally:
        dist.destroy_process_group()


def test_replica_reductions_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort(key=lambda r: r["rank"])
    assert [r["first"] for r in out] == [100, 164]
    assert all(r["n"] == 64 for r in out)
    assert all(r["tmax"] == 2.0 for r in out)
    assert all(r["esum"] == 3000.0 for r in out)
    assert all(abs(r["rate"] - 1500.0) < 1e-9 for r in out)


def test_shard_without_weak_scaling():
    from sygraph_b200 import replicas
    parts = [replicas.shard(np.arange(10), r, 3) for r in range(3)]
    assert np.array_equal(np.concatenate(parts), np.arange(10))
    with pytest.raises(ValueError):
        replicas.shard(np.arange(10), 0, 2, per_rank=6)
