"""Shared helpers of the test suite: random physical states, one reference
step through the oracle, error measures."""
from __future__ import annotations

import numpy as np


def random_q(o, rng, rho=(0.5, 2.0), vel=(-0.5, 0.5), pres=(0.5, 2.0)):
    """Random conserved state in the reference layout for oracle `o`."""
    q = o.zeros_q()
    sh = q.shape[:3]
    r = rng.uniform(*rho, sh)
    v = rng.uniform(*vel, sh + (3,))
    p = rng.uniform(*pres, sh)
    if o.p.ny == 1:
        v[..., 1] = 0.0
    if o.p.nz == 1:
        v[..., 2] = 0.0
    q[..., 0] = r
    q[..., 1:4] = r[..., None] * v
    q[..., 4] = 0.5 * r * (v ** 2).sum(-1) + p / o.d.g1
    q[..., 5] = p / r ** o.d.g1
    return q


def oracle_step(o, q):
    """One step of main.f90:111-155 on a copy of q; returns (q_new, dt, t)."""
    w = np.zeros(o.shape_w)
    evo = np.zeros(o.shape_evo)
    s = np.zeros(o.shape_s)
    o.primitive(w, q)
    o.bound(w)
    dt = o.hydrostep(w, 1e99)
    go, t, dt = o.updatetime(o.p.tstart, dt)
    if o.p.secondorder:
        o.compevo(w, evo, s, dt)
    q2 = q.copy()
    o.sweep(w, q2, evo, s, dt)
    return q2, dt, t


def rel_l1(a, b):
    """Relative L1 difference sum|a-b| / sum|b| per field (last axis)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, a.shape[-1])
    b = np.asarray(b, dtype=np.float64).reshape(-1, b.shape[-1])
    num = np.abs(a - b).sum(axis=0)
    den = np.abs(b).sum(axis=0)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def oracle_tube_task(task):
    """One 1D tube through the oracle's time loop (spawned worker process)."""
    from oracle.oracle import run_tube
    return run_tube(task)
