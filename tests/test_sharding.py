"""Multi-rank path on CPU: two gloo ranks shard independent tubes by work,
advance their shards (CPU oracle standing in for the GPU batch), reduce the
timing with max over ranks and gather; the gathered result equals the
single-process run, and the split is complete, disjoint and balanced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import evora_b200 as ev
from evora_b200 import sharding


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run_tubes_cpu(lengths, q, kw):
    from oracle.oracle import Oracle, make_params
    out, off = [], 0
    for n in lengths:
        o = Oracle(make_params(nx=n, ny=1, nz=1, **kw))
        qq = q[off:off + n].reshape(1, 1, n, 6).copy()
        o.run(qq, 1 << 30)
        out.append(qq.reshape(n, 6))
        off += n
    return np.concatenate(out) if out else np.zeros((0, 6))


KW = dict(g=5 / 3, cfl=0.8, boundtype=1, tend=0.01)


def _worker(rank, world, port, lengths, q, result_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    work = sharding.tube_work(lengths, q)
    shards = sharding.shard_by_work(work, world)
    sel_len, sel_q = sharding.pack(lengths, q, shards[rank])
    part = _run_tubes_cpu(sel_len, sel_q, KW)
    t = sharding.max_over_ranks(float(rank + 1))
    full = sharding.gather_to_rank0(lengths, shards, part, rank, world)
    if rank == 0:
        np.savez(result_path, full=full, tmax=t)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_by_work_is_complete_and_balanced():
    rng = np.random.default_rng(0)
    work = list(rng.uniform(1, 100, 500))
    for world in (1, 2, 3, 8):
        shards = sharding.shard_by_work(work, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(500))
        loads = [sum(work[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(work)


def test_two_gloo_ranks_match_single_process(tmp_path):
    lengths, q = ev.ic.random_tubes(9, seed=4, nmin=16, nmax=120)
    ref = _run_tubes_cpu(lengths, q, KW)
    path = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(2, _free_port(), lengths, q, path), nprocs=2, join=True,
                       start_method="spawn")
    res = np.load(path)
    assert float(res["tmax"]) == 2.0
    np.testing.assert_array_equal(res["full"], ref)


def test_assign_online_is_deterministic_and_balanced():
    """Serving requests go, in arrival order, to the rank with the least
    estimated work so far: every request has exactly one rank, every rank
    computes the same assignment, and the loads end within the largest
    single request of each other."""
    rng = np.random.default_rng(3)
    shapes = [(1, 1, int(n), 6) for n in rng.integers(128, 8193, 300)]
    shapes += [(1, int(m), int(m), 6) for m in 16 * rng.integers(4, 65, 150)]
    shapes += [(int(m), int(m), int(m), 6) for m in 16 * rng.integers(2, 9, 50)]
    order = rng.permutation(len(shapes))
    work = [sharding.request_work(shapes[i], 0.05) for i in order]
    for world in (1, 2, 3, 8):
        a = sharding.assign_online(work, world)
        assert a == sharding.assign_online(list(work), world)
        assert len(a) == len(work) and set(a) <= set(range(world))
        load = np.zeros(world)
        for w, r in zip(work, a):
            load[r] += w
        assert load.max() - load.min() <= max(work) + 1e-9
    # cells x the largest edge (the steps to a fixed end time), x tend
    assert sharding.request_work((1, 1, 4096, 6)) == 4096.0 * 4096
    assert sharding.request_work((16, 16, 16, 6), 0.5) == 4096.0 * 16 * 0.5


def _serving_worker(rank, world, port, work, result_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    owner = sharding.assign_online(work, world)
    mine = [i for i, r in enumerate(owner) if r == rank]
    parts = sharding.gather_objects((rank, mine, sum(work[i] for i in mine)), rank, world)
    if rank == 0:
        np.savez(result_path, ranks=[p[0] for p in parts], loads=[p[2] for p in parts],
                 idx=np.concatenate([np.asarray(p[1], dtype=np.int64) for p in parts]))
    dist.barrier()
    dist.destroy_process_group()


def test_serving_requests_split_over_two_gloo_ranks(tmp_path):
    """Two gloo ranks assign the same request list independently and gather
    their shares on rank 0: every request is served exactly once."""
    rng = np.random.default_rng(4)
    work = [float(w) for w in rng.uniform(1, 1000, 400)]
    path = str(tmp_path / "serving.npz")
    mp.spawn(_serving_worker, args=(2, _free_port(), work, path), nprocs=2, join=True)
    r = np.load(path)
    assert list(r["ranks"]) == [0, 1]
    assert sorted(r["idx"].tolist()) == list(range(len(work)))
    assert abs(r["loads"][0] - r["loads"][1]) <= max(work)
