"""The multi-GPU bench path on CPU: two gloo ranks shard the sweep without
overlap and reduce (max time, summed converged pairs) as bench.py does."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    from qdsim_b200 import workloads as W
    first = bench.shard_first(rank, 3)
    ids = list(range(first, first + 3))
    # the shard bench.py builds is exactly dots first .. first+2 of the sweep
    for i, d in zip(ids, W.sweep_batch(3, first=first)):
        ref = W.sweep_dot(i)
        assert d.mesh.nx == ref.mesh.nx and (d.V == ref.V).all()
    ms, conv = bench.reduce_over_ranks(10.0 + rank, 8.0 * (rank + 1), world, torch.device("cpu"))
    out.put((rank, ids, ms, conv))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_and_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ids0, ms0, c0), (r1, ids1, ms1, c1) = res
    assert set(ids0).isdisjoint(ids1)            # no dot solved twice
    assert ms0 == ms1 == 11.0                    # max over ranks
    assert c0 == c1 == 8.0 + 16.0                # pairs summed
