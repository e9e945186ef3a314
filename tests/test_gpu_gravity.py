"""Self-gravity on the GPU (gravitation.f90, non-comoving) against the numpy
restatement (oracle/gravity_oracle.py): the drop-in gravpotential and
gravintegration, and grids whose steps add the gravity substep after the
hydro update.  FFTW 2.1.5 is not part of the reference tree, so the
potential has no bit-level reference: it must agree with numpy's FFT to
round-off and invert the discrete Laplacian."""
import numpy as np
import pytest
import torch

import evora_b200 as ev
from helpers import oracle_step
from oracle import gravity_oracle as go
from oracle.oracle import Oracle, make_params

pytestmark = pytest.mark.gpu

SHAPES = [(16, 12, 10), (24, 20, 1), (64, 1, 1)]
IDS = ["3d", "2d", "1d"]


def dense_state(p, seed=0):
    """Densities of order 1e6 so that the gravitational terms (4 pi G =
    8.4e-7 in code units) are not lost below the hydro state's rounding."""
    rng = np.random.default_rng(seed)
    sh = (p.nz, p.ny, p.nx)
    r = 1e6 * rng.uniform(0.5, 2.0, sh)
    v = rng.uniform(-0.5, 0.5, sh + (3,))
    if p.ny == 1:
        v[..., 1] = 0
    if p.nz == 1:
        v[..., 2] = 0
    pr = 1e6 * rng.uniform(0.5, 2.0, sh)
    g1 = ev.derived(p).g1
    q = np.empty(sh + (6,))
    q[..., 0] = r
    q[..., 1:4] = r[..., None] * v
    q[..., 4] = 0.5 * r * (v ** 2).sum(-1) + pr / g1
    q[..., 5] = pr / r ** g1
    return q


@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_dropin_gravpotential_matches_numpy(cuda_device, shape):
    nx, ny, nz = shape
    p = ev.default_params(nx=nx, ny=ny, nz=nz, gravity=1)
    d = ev.derived(p)
    q = dense_state(p, seed=nx)
    phi = np.zeros((nz, ny, nx), np.complex128)
    ev.DropIn(p).gravpotential(q, phi)
    ref = go.gravpotential(q, d.dx)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(phi.real - ref)) <= 1e-12 * scale
    assert np.all(phi.imag == 0.0)
    src = go.FOURPIG * (q[..., 0] - q[..., 0].mean())
    assert np.max(np.abs(go.laplacian(phi.real, d.dx) - src)) < 1e-6 * np.max(np.abs(src))


@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_dropin_gravintegration_matches_numpy(cuda_device, shape):
    nx, ny, nz = shape
    p = ev.default_params(nx=nx, ny=ny, nz=nz, gravity=1)
    d = ev.derived(p)
    q = dense_state(p, seed=nx + 1)
    phi = np.ascontiguousarray(np.random.default_rng(5).normal(size=(nz, ny, nx)) + 0j)
    out = q.copy()
    ev.DropIn(p).gravintegration(out, phi, 1e-3)
    ref = go.gravintegration(q, phi.real, 1e-3, d.dx, d.dy, d.dz)
    np.testing.assert_array_equal(out[..., 0], q[..., 0])
    np.testing.assert_array_equal(out[..., 5], q[..., 5])
    np.testing.assert_allclose(out, ref, rtol=1e-15, atol=0)


@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_grid_step_with_gravity_matches_oracle(cuda_device, shape):
    # one step = the oracle's hydro step (bit-exact in strict FP64) followed
    # by gravpotential + gravintegration on the updated state
    nx, ny, nz = shape
    kw = dict(nx=nx, ny=ny, nz=nz, boundtype=2, cfl=0.4, tend=10.0)
    p = ev.default_params(**kw, gravity=1)
    o = Oracle(make_params(**kw))
    q0 = dense_state(p, seed=7)
    q1, dt, _ = oracle_step(o, q0)
    d = ev.derived(p)
    ref = go.gravintegration(q1, go.gravpotential(q1, d.dx), dt, d.dx, d.dy, d.dz)
    with ev.Grid(p, ev.FP64, ev.STRICT | ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        g.step(1)
        t = g.time()
        q = g.get_q()
    assert t["dt"] == dt and t["k"] == 1
    np.testing.assert_array_equal(q[..., 0], q1[..., 0])
    for f in range(6):   # the potentials differ at FFT round-off
        assert np.max(np.abs(q[..., f] - ref[..., f])) <= 1e-12 * np.max(np.abs(ref[..., f])), f
    # gravity changed the momenta: the comparison is not vacuous
    assert np.max(np.abs(ref[..., 1:4] - q1[..., 1:4])) > 1e-9 * np.max(np.abs(q1[..., 1:4]))


@pytest.mark.parametrize("precision", [ev.FP64, ev.FP32])
def test_grid_with_gravity_graphs_equal_single_steps(cuda_device, precision):
    p = ev.default_params(nx=32, ny=24, nz=16, boundtype=2, cfl=0.4, tend=10.0, gravity=1)
    q0 = dense_state(p, seed=9)
    with ev.Grid(p, precision) as a:
        a.set_q(q0)
        for _ in range(6):
            a.step(1)
        qa, ta = a.get_q(), a.time()
    stream = torch.cuda.Stream()
    with ev.Grid(p, precision, stream=stream) as b:
        b.set_q(q0)
        b.step(6)                     # graph-captured steps (cuFFT inside)
        qb, tb = b.get_q(), b.time()
    assert ta == tb
    np.testing.assert_array_equal(qa, qb)


def test_fp32_gravity_close_to_fp64(cuda_device):
    p = ev.default_params(nx=32, ny=32, nz=32, boundtype=2, cfl=0.4, tend=10.0, gravity=1)
    q0 = dense_state(p, seed=11)
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(p, prec) as g:
            g.set_q(q0)
            g.step(5)
            out[prec] = g.get_q()
    a, b = out[ev.FP32][..., 0], out[ev.FP64][..., 0]
    assert np.abs(a - b).sum() / np.abs(b).sum() < 1e-5
