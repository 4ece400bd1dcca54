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


def _lpt_worker(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from qdsim_b200 import batch as B
    from qdsim_b200 import workloads as W
    dots = [W.sweep_dot(i, nx=nx) for i, nx in enumerate([40, 200, 60, 120, 80, 240, 44, 90])]
    idx, mine = B.shard_dots(dots, rank, world)
    # stand-in per-dot results (k = 3 "eigenvalues" that name their dot)
    local = np.stack([np.full(3, 10.0 * i) + np.arange(3) for i in idx])
    full = B.gather_by_index(local, idx, len(dots))
    out.put((rank, idx.tolist(), [d.mesh.nx for d in mine], full.tolist(),
             [B.dot_cost(d) for d in dots]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_cost_balanced_shards_and_gather():
    """A fixed set of dots split over two gloo ranks by predicted cost: the
    shards are disjoint and cover every dot, the heavier one is within the
    LPT bound, and gather_by_index gives every rank all results in dot order."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_lpt_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, i0, nx0, f0, cost), (_, i1, nx1, f1, _) = res
    assert sorted(i0 + i1) == list(range(8)) and set(i0).isdisjoint(i1)
    loads = [sum(cost[i] for i in i0), sum(cost[i] for i in i1)]
    bound = max(sum(cost) / 2, max(cost))
    assert max(loads) <= 4 / 3 * bound
    want = [[10.0 * i, 10.0 * i + 1, 10.0 * i + 2] for i in range(8)]
    assert f0 == want and f1 == want


def test_partition_by_cost_rules():
    import numpy as np
    from qdsim_b200 import batch as B
    g = B.partition_by_cost([5, 4, 3, 3, 3], 2)
    assert [a.tolist() for a in g] == [[0, 3], [1, 2, 4]]      # loads 8 and 10
    g = B.partition_by_cost([1.0] * 5, 3)
    assert [a.tolist() for a in g] == [[0, 3], [1, 4], [2]]
    assert [a.tolist() for a in B.partition_by_cost([], 2)] == [[], []]
    with pytest.raises(ValueError):
        B.partition_by_cost([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        B.partition_by_cost([1.0], 0)
    with pytest.raises(ValueError):
        B.gather_by_index(np.zeros((2, 3)), [0, 0], 2)             # repeated item
    with pytest.raises(ValueError):
        B.gather_by_index(np.zeros((1, 3)), [0], 2)                # item 1 missing
    np.testing.assert_array_equal(B.gather_by_index(np.array([[2.0], [1.0]]), [1, 0], 2),
                                  [[1.0], [2.0]])
