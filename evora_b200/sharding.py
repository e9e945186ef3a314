"""Sharding of independent work across ranks (one process per GPU).

A single grid is not decomposed (one grid per GPU; more GPUs run replicas).
Independent tubes or requests shard by whole units: `shard_by_work` assigns
each unit to a rank, largest estimated work first, always to the rank with
the least work so far (LPT), so the ranks finish together; serving requests,
which arrive over time, go one by one to the least-loaded rank
(`assign_online`).  No data moves between ranks during the run.  The helpers below gather the per-rank
results and reduce timings (max over ranks) with torch.distributed; they
work with the NCCL backend on GPUs and with gloo on CPU (tests)."""
from __future__ import annotations

import heapq

import numpy as np


def tube_work(lengths, q=None, gamma=5.0 / 3.0):
    """Estimated work of each tube: n^2 * max(|u| + a) of its initial state
    (steps to a fixed end time grow with n * max speed), n^2 without q."""
    lengths = [int(n) for n in lengths]
    if q is None:
        return [float(n) * n for n in lengths]
    out, off = [], 0
    g1 = gamma - 1.0
    for n in lengths:
        c = q[off:off + n]
        rho = c[:, 0]
        u = c[:, 1] / rho
        p = g1 * (c[:, 4] - 0.5 * (c[:, 1] ** 2 + c[:, 2] ** 2 + c[:, 3] ** 2) / rho)
        s = np.abs(u) + np.sqrt(np.maximum(gamma * p / rho, 0.0))
        out.append(float(n) * n * float(s.max()))
        off += n
    return out


def shard_by_work(work, world):
    """Per-rank lists of unit indices (LPT: largest first to the least
    loaded rank).  Deterministic: every rank computes the same split."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(s) for s in shards]


def request_work(shape, tend=1.0):
    """Estimated work of a serving request on a state of `shape` (nz, ny,
    nx, nf) run to time tend: cells x steps, the steps growing with the
    largest edge length (a fixed CFL number over cells of size 1/n)."""
    cells = int(np.prod(shape[:-1]))
    return float(cells) * max(shape[:-1]) * float(tend)


def assign_online(work, world):
    """Per-request rank for requests arriving in order, each to the rank with
    the least estimated work assigned so far (ties to the lowest rank): the
    dispatch a front end makes without knowing later arrivals.  Deterministic,
    so every rank computes the same assignment from the same request list."""
    load = [0.0] * world
    out = []
    for w in work:
        r = min(range(world), key=lambda k: (load[k], k))
        out.append(r)
        load[r] += float(w)
    return out


def gather_objects(obj, rank, world):
    """Every rank's `obj` on rank 0, in rank order (None elsewhere)."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    objs = [None] * world if rank == 0 else None
    dist.gather_object(obj, objs, dst=0)
    return objs


def pack(lengths, q, indices):
    """Lengths and concatenated states of the selected tubes."""
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    sel_len = [int(lengths[i]) for i in indices]
    parts = [q[offs[i]:offs[i + 1]] for i in indices]
    return sel_len, (np.ascontiguousarray(np.concatenate(parts)) if parts else np.zeros((0, q.shape[1])))


def unpack_into(out, lengths, indices, q_part):
    """Writes the packed results of `indices` back into the full array."""
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    k = 0
    for i in indices:
        n = int(lengths[i])
        out[offs[i]:offs[i + 1]] = q_part[k:k + n]
        k += n
    return out


def max_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_rank0(lengths, shards, q_part, rank, world):
    """Collects every rank's packed tube results on rank 0 (object gather:
    results only, after the run).  Returns the full array on rank 0."""
    import torch.distributed as dist
    if world == 1:
        full = np.zeros((int(sum(lengths)), q_part.shape[1]))
        return unpack_into(full, lengths, shards[0], q_part)
    objs = [None] * world if rank == 0 else None
    dist.gather_object(q_part, objs, dst=0)
    if rank != 0:
        return None
    full = np.zeros((int(sum(lengths)), q_part.shape[1]))
    for r in range(world):
        unpack_into(full, lengths, shards[r], objs[r])
    return full
