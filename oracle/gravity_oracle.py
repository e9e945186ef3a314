"""numpy restatement of the reference's self-gravity -- TEST INFRASTRUCTURE
ONLY (used by tests/ as the checker of evora_b200/csrc/gravity.cu; the
product never imports it).

Follows the non-comoving branch of gravitation.f90:
  gravpotential   26-53   source grav (rho - mean rho), forward FFT,
  multigreen      55-84   times green / n3 with green = -h2 / (sin^2(kfx/2 kx)
                          + sin^2(kfy/2 ky) + sin^2(kfz/2 kz)), 0 at k = 0,
                          backward FFT (unnormalised, FFTW's convention)
  gravintegration 170-194 and grav_force 196-243 (periodic centred
                          differences)
with the constants of compparameter (parameter.f90:219, 240, 254-263) and
kvalue (comp.f90:241-252).  The FFTs are numpy's (pocketfft) instead of the
reference's FFTW 2.1.5, which is not part of the reference tree: the
potential agrees with any correct FFT to rounding, not bit for bit.
"""
from __future__ import annotations

import numpy as np

FOURPIG = 8.38553911e-7          # global.f90:101
PI = float(np.float32(3.1415927))  # module global's pi, a default-real literal


def kvalue(i: int, n: int, nyq: int) -> float:
    return float(i - 1) if i <= nyq else -float(n - (i - 1))


def sin2_table(n: int) -> np.ndarray:
    nyq = max(n // 2, 1)
    kf = 2.0 * PI / n
    kf2 = kf * 0.5
    return np.array([np.sin(kf2 * kvalue(i, n, nyq)) ** 2 for i in range(1, n + 1)])


def green(nx: int, ny: int, nz: int, dx: float) -> np.ndarray:
    """multigreen's factor on the full spectrum, C shape (nz, ny, nx)."""
    h2 = dx * dx / 4.0
    sx, sy, sz = sin2_table(nx), sin2_table(ny), sin2_table(nz)
    den = (sx[None, None, :] + sy[None, :, None]) + sz[:, None, None]
    with np.errstate(divide="ignore"):
        g = -h2 / den
    g[0, 0, 0] = 0.0
    return g


def gravpotential(q: np.ndarray, dx: float, comoving=None) -> np.ndarray:
    """q of C shape (nz, ny, nx, 6) -> real potential, C shape (nz, ny, nx).
    comoving = (cosmo, omega0, fb) takes the comoving source
    cosmo * grav * (rho / fb - 1) with grav = 1.5 omega0 (gravitation.f90:36-37,
    parameter.f90:236-238)."""
    nz, ny, nx = q.shape[:3]
    rho = q[..., 0]
    if comoving is not None:
        cosmo, omega0, fb = comoving
        src = cosmo * (1.5 * omega0) * (rho / fb - 1.0)
    else:
        mean = rho.sum() / (nx * ny * nz)
        src = FOURPIG * (rho - mean)
    spec = np.fft.fftn(src)
    spec = spec / float(nx * ny * nz) * green(nx, ny, nz, dx)
    # FFTW's backward transform is unnormalised: n3 * numpy's ifftn
    return (np.fft.ifftn(spec) * (nx * ny * nz)).real


def forces(phi: np.ndarray, dx: float, dy: float, dz: float) -> tuple:
    nz, ny, nx = phi.shape
    f1 = -(np.roll(phi, -1, 2) - np.roll(phi, 1, 2)) * (0.5 / dx) if nx != 1 else np.zeros_like(phi)
    f2 = -(np.roll(phi, -1, 1) - np.roll(phi, 1, 1)) * (0.5 / dy) if ny != 1 else np.zeros_like(phi)
    f3 = -(np.roll(phi, -1, 0) - np.roll(phi, 1, 0)) * (0.5 / dz) if nz != 1 else np.zeros_like(phi)
    return f1, f2, f3


def gravintegration(q: np.ndarray, phi: np.ndarray, dt: float, dx: float, dy: float, dz: float) -> np.ndarray:
    q = q.copy()
    f1, f2, f3 = forces(phi, dx, dy, dz)
    q[..., 4] = q[..., 4] + dt * (q[..., 1] * f1 + q[..., 2] * f2 + q[..., 3] * f3)
    q[..., 1] = q[..., 1] + dt * q[..., 0] * f1
    q[..., 2] = q[..., 2] + dt * q[..., 0] * f2
    q[..., 3] = q[..., 3] + dt * q[..., 0] * f3
    return q


def laplacian(phi: np.ndarray, dx: float) -> np.ndarray:
    """The 7-point Laplacian (cubic cells) that multigreen's factor inverts:
    its eigenvalue for mode k is -4 sum_d sin^2(pi k_d / n_d) / dx^2 = 1 / (green n3 / n3)."""
    lap = np.zeros_like(phi)
    for ax in range(3):
        if phi.shape[ax] > 1:
            lap += np.roll(phi, -1, ax) - 2.0 * phi + np.roll(phi, 1, ax)
    return lap / (dx * dx)
