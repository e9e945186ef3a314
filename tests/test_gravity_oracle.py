"""The numpy restatement of the reference's self-gravity (oracle/
gravity_oracle.py) against what its Poisson solve must satisfy: the
potential inverts the 7-point Laplacian (with module global's single-
precision pi in the Green's function, hence ~1e-7 rather than round-off),
has zero mean, and a single Fourier mode gives the analytic amplitude."""
import numpy as np
import pytest

from oracle import gravity_oracle as go


def field(shape, seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    q = np.zeros(shape + (6,))
    q[..., 0] = scale * rng.uniform(0.5, 2.0, shape)
    return q


@pytest.mark.parametrize("shape", [(8, 12, 16), (1, 10, 14), (1, 1, 32)], ids=["3d", "2d", "1d"])
def test_potential_inverts_laplacian(shape):
    nz, ny, nx = shape
    dx = 1.0 / nx
    q = field(shape, seed=nx)
    phi = go.gravpotential(q, dx)
    src = go.FOURPIG * (q[..., 0] - q[..., 0].mean())
    lap = go.laplacian(phi, dx)
    assert np.max(np.abs(lap - src)) < 1e-6 * np.max(np.abs(src))
    assert abs(phi.mean()) < 1e-12 * np.max(np.abs(phi))


def test_single_mode_amplitude():
    n, k, amp = 32, 3, 0.1
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    q = np.zeros((1, 1, n, 6))
    q[0, 0, :, 0] = 1.0 + amp * np.cos(2 * np.pi * k * x)
    phi = go.gravpotential(q, dx)[0, 0]
    s2 = np.sin(go.PI * k / n) ** 2
    expect = -go.FOURPIG * amp * np.cos(2 * np.pi * k * x) * (dx * dx / 4.0) / s2
    np.testing.assert_allclose(phi, expect, rtol=0, atol=1e-12 * np.max(np.abs(expect)))


def test_integration_uses_old_momentum_for_energy():
    q = field((4, 4, 4), seed=3)
    q[..., 1:4] = 0.3
    q[..., 4] = 5.0
    phi = np.random.default_rng(4).normal(size=(4, 4, 4))
    out = go.gravintegration(q, phi, 0.01, 0.25, 0.25, 0.25)
    f1, f2, f3 = go.forces(phi, 0.25, 0.25, 0.25)
    np.testing.assert_allclose(out[..., 4], 5.0 + 0.01 * 0.3 * (f1 + f2 + f3), rtol=1e-15)
    np.testing.assert_allclose(out[..., 1], 0.3 + 0.01 * q[..., 0] * f1, rtol=1e-15)
