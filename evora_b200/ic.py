"""Initial conditions in the reference layout q (nz, ny, nx, 6), built on the
host in FP64 (the reference builds them on the host too, ic(q) in ic/*.f90).

Cell centres follow coordinates() (comp.f90:150-162): x = x0 + (ix-1) dx.
"""
from __future__ import annotations

import numpy as np

from .hydro import EvoraParams, derived


def _centres(p: EvoraParams):
    d = derived(p)
    x = d.x0 + np.arange(p.nx, dtype=np.float64) * d.dx
    y = d.y0 + np.arange(p.ny, dtype=np.float64) * d.dy
    z = d.z0 + np.arange(p.nz, dtype=np.float64) * d.dz
    return d, x, y, z


def shocktube(p: EvoraParams, dl=1.0, ul=0.0, pl=1.0, dr=0.125, ur=0.0, pr=0.1, x_diss=0.5, direction=1):
    """ic(q) of ic/shocktube.f90:59-100: a Riemann problem split at x_diss
    along direction 1, 2 or 3."""
    if direction not in (1, 2, 3):
        raise ValueError("direction must be 1, 2 or 3")
    d, x, y, z = _centres(p)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    coord = (X, Y, Z)[direction - 1]
    left = coord < x_diss
    rho = np.where(left, dl, dr)
    u = np.where(left, ul, ur)
    pres = np.where(left, pl, pr)
    q = np.zeros((p.nz, p.ny, p.nx, 6))
    q[..., 0] = rho
    q[..., direction] = rho * u
    q[..., 4] = 0.5 * rho * (u * u) + pres / d.g1
    q[..., 5] = pres / rho ** d.g1
    return q


def kh2d(p: EvoraParams):
    """ic(q) of ic/kevinhelmholtz.f90:40-69 (the reference's 2D shear layer;
    pi and the literals 0.1, 0.05 are single precision there)."""
    d, x, y, z = _centres(p)
    pi = float(np.float32(3.1415927))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.abs(Y - 0.5)
    inside = r <= 0.25
    rho = np.where(inside, 2.0, 1.0)
    u = np.where(inside, 0.5, -0.5)
    v = float(np.float32(0.1)) * np.sin(4 * pi * X) * (
        np.exp(-((Y - 0.25) * (Y - 0.25)) / float(np.float32(0.05)))
        + np.exp(-((Y - 0.75) * (Y - 0.75)) / float(np.float32(0.05))))
    pres = 2.5
    q = np.zeros((p.nz, p.ny, p.nx, 6))
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 4] = 0.5 * rho * ((u * u) + (v * v)) + pres / (d.g - 1)
    q[..., 5] = pres / rho ** (d.g - 1)
    return q


def _splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


def kh3d_phases(seed=42):
    """Phases phi_k = 2 pi u_k, u_k from the top 53 bits of SplitMix64(seed)."""
    st = seed & 0xFFFFFFFFFFFFFFFF
    out = []
    for _ in range(4):
        st, r = _splitmix64(st)
        out.append(6.283185307179586 * ((r >> 11) * 2.0 ** -53))
    return out


def kh3d(p: EvoraParams, seed=42, amp=0.01):
    """The 3D Kelvin-Helmholtz workload (256^3 periodic, gamma = 5/3 in the
    benchmark): slab |y - 0.5| < 0.25 with rho = 2, vx = +0.5; outside
    rho = 1, vx = -0.5; p = 2.5; vz = 0;
    vy = amp * sum_{k=1..4} sin(2 pi k x + phi_k) with seeded phases."""
    d, x, y, z = _centres(p)
    phi = kh3d_phases(seed)
    twopi = 6.283185307179586
    vx_line = np.zeros_like(x)
    for k in range(4):
        vx_line = vx_line + np.sin(twopi * float(k + 1) * x + phi[k])
    vy_line = amp * vx_line
    inside = np.abs(y - 0.5) < 0.25
    rho_y = np.where(inside, 2.0, 1.0)
    u_y = np.where(inside, 0.5, -0.5)
    rho = np.broadcast_to(rho_y[None, :, None], (p.nz, p.ny, p.nx))
    u = np.broadcast_to(u_y[None, :, None], (p.nz, p.ny, p.nx))
    v = np.broadcast_to(vy_line[None, None, :], (p.nz, p.ny, p.nx))
    q = np.zeros((p.nz, p.ny, p.nx, 6))
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 4] = 0.5 * rho * ((u * u) + (v * v)) + 2.5 / d.g1
    q[..., 5] = 2.5 / rho ** d.g1
    return q


def random_tubes(ntubes, seed=7, nmin=128, nmax=4096, gamma=5.0 / 3.0):
    """The batched Riemann-problem workload: tube lengths uniform in
    [nmin, nmax]; left/right rho log-uniform in [0.1, 10], p log-uniform in
    [0.01, 10], v uniform in [-1, 1]; interface uniform in [0.3, 0.7].
    Returns (lengths, q) with q of shape (sum lengths, 6) in the reference
    layout, tubes concatenated, built like ic/shocktube.f90:59-100."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(nmin, nmax + 1, ntubes)
    rho = np.exp(rng.uniform(np.log(0.1), np.log(10.0), (ntubes, 2)))
    pre = np.exp(rng.uniform(np.log(0.01), np.log(10.0), (ntubes, 2)))
    vel = rng.uniform(-1.0, 1.0, (ntubes, 2))
    xd = rng.uniform(0.3, 0.7, ntubes)
    g1 = gamma - 1.0
    parts = []
    for i in range(ntubes):
        n = int(lengths[i])
        dx = 1.0 / n
        x = dx / 2 + np.arange(n) * dx
        left = x < xd[i]
        d = np.where(left, rho[i, 0], rho[i, 1])
        u = np.where(left, vel[i, 0], vel[i, 1])
        p = np.where(left, pre[i, 0], pre[i, 1])
        q = np.zeros((n, 6))
        q[:, 0] = d
        q[:, 1] = d * u
        q[:, 4] = 0.5 * d * (u * u) + p / g1
        q[:, 5] = p / d ** g1
        parts.append(q)
    return [int(x) for x in lengths], np.ascontiguousarray(np.concatenate(parts))
