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


def _kvalue(n):
    """kvalue (comp.f90:241-252) over the FFT index order: 0, 1, ..., then
    the negative wavenumbers above the Nyquist index max(n/2, 1)."""
    nyq = max(n // 2, 1)
    i = np.arange(1, n + 1)
    return np.where(i <= nyq, i - 1, -(n - (i - 1))).astype(np.float64)


def _sin2(n):
    """sin^2(kf/2 k) of multigreen (gravitation.f90:55-84), kf = 2 pi / n with
    module global's single-precision pi (global.f90:98)."""
    pi = float(np.float32(3.1415927))
    return np.sin((2.0 * pi / n) * 0.5 * _kvalue(n)) ** 2


def cosmo_zeldovich(p: EvoraParams, seed=5, slope=-2.0, sigma=0.05, temp_k=100.0):
    """A comoving box in the Zel'dovich approximation, built as ic/cosmo.f90
    builds it (25-180) with a seeded power law in place of its tabulated
    spectrum:

      white noise / sqrt(n3) -> FFT -> times sqrt(P(k)), P = k^slope with
      k = |k| 2 pi / box (multipower, gravitation.f90:90-168, k = 0 removed)
      -> inverse FFT -> density contrast delta, scaled to rms `sigma`;
      rho = fb (1 + delta) (the baryon fraction applied as ic/pancake.f90:89
      does, so that the comoving source rho/fb - 1 is delta);
      phi from delta with multigreen's discrete Green's function;
      v = fpeebles adot/a (-grad phi), centred periodic differences
      (grav_force, gravitation.f90:196-243; peebles, cosmology.f90:76-97);
      T = temp_k (rho/fb)^(g-1) Kelvin, p = rho T / temp0 at the start
      (press2temp, comp.f90:87-102).

    p must enable supercomoving; the FFTs are numpy's (real-to-complex, which
    is the reference's complex transform of a real field).  Returns q of shape
    (nz, ny, nx, 6)."""
    import ctypes

    from . import _native
    from ._native import check
    from .hydro import DropIn
    if not p.supercomoving:
        raise ValueError("cosmo_zeldovich needs supercomoving = 1")
    d = derived(p)
    nz, ny, nx = p.nz, p.ny, p.nx
    n3 = nx * ny * nz
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((nz, ny, nx)) / np.sqrt(float(n3))
    spec = np.fft.rfftn(white)
    kx, ky, kz = _kvalue(nx)[: nx // 2 + 1], _kvalue(ny), _kvalue(nz)
    k2 = (kx[None, None, :] ** 2 + ky[None, :, None] ** 2) + kz[:, None, None] ** 2
    kk = np.sqrt(k2) * (2.0 * np.pi / p.box)
    with np.errstate(divide="ignore"):
        pk = np.where(k2 > 0, kk ** (0.5 * slope), 0.0)
    delta = np.fft.irfftn(spec * pk, s=(nz, ny, nx), axes=(0, 1, 2))
    delta *= sigma / np.sqrt(np.mean(delta * delta))
    rho = p.fb * (1.0 + delta)
    green = np.zeros_like(k2)
    den = (_sin2(nx)[: nx // 2 + 1][None, None, :] + _sin2(ny)[None, :, None]) + _sin2(nz)[:, None, None]
    green[k2 > 0] = -(d.dx * d.dx / 4.0) / den[k2 > 0]
    phi = np.fft.irfftn(np.fft.rfftn(delta) * green, s=(nz, ny, nx), axes=(0, 1, 2))
    drop = DropIn(p)
    s = drop.cosmostart()
    vscale = drop.peebles(s) * s["cosmodot"] / s["cosmo"]
    vel = np.zeros((nz, ny, nx, 3))
    for ax, (n, h) in enumerate(((nx, d.dx), (ny, d.dy), (nz, d.dz))):
        if n > 1:
            axis = 2 - ax
            vel[..., ax] = -vscale * (np.roll(phi, -1, axis) - np.roll(phi, 1, axis)) * (0.5 / h)
    u = _native.EvoraUnits()
    check(_native.lib().evora_compunits(ctypes.byref(p), None, ctypes.byref(u)), "compunits")
    temp = temp_k * (rho / p.fb) ** d.g1
    if p.chemistry:
        # temp2press (comp.f90:104-119) with the neutral abundances initchem
        # sets: T sum(n) / temp0, n(H) = rho rhoH / mH, n(He) = rho rhoHe / mHe
        mh, mhe = float(np.float32(1.00794)), float(np.float32(4.002602))
        pres = temp * (rho * (p.rhoh / mh) + rho * (p.rhohe / mhe)) / u.temp0
    else:
        pres = rho * temp / u.temp0
    q = np.zeros((nz, ny, nx, 12 if p.chemistry else 6))
    q[..., 0] = rho
    q[..., 1:4] = rho[..., None] * vel
    q[..., 4] = 0.5 * rho * (vel ** 2).sum(-1) + pres / d.g1
    q[..., 5] = pres / rho ** d.g1
    if p.chemistry:
        drop.initchem(q)   # q(7:12): fully neutral (initchem, chemistry.f90:26-70)
    return q
