"""The CPU oracle against known answers: the exact Riemann solution of the
Sod problem (Toro ch. 4), conservation in periodic boxes, and the direction
symmetry of the shocktube IC (ic/shocktube.f90:64-90)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, make_params
import exact_riemann as ex
from helpers import oracle_step, random_q


def sod(n, **kw):
    p = make_params(nx=n, ny=1, nz=1, g=1.4, cfl=0.8, boundtype=1, tend=0.2, **kw)
    o = Oracle(p)
    q = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1)
    r = o.run(q, 100000)
    x = o.d.x0 + np.arange(n) * o.d.dx
    e = ex.sample(x, r["t"], 0.5, (1, 0, 1), (0.125, 0, 0.1), 1.4)
    return q, r, e


def test_sod_matches_exact_solution_and_converges():
    errs = []
    for n in (128, 512):
        q, r, e = sod(n)
        assert r["status"] == 0 and not r["go"]
        assert r["t"] == pytest.approx(0.2, abs=0, rel=0)
        rho = q[0, 0, :, 0]
        errs.append(np.mean(np.abs(rho - e[0])))
    assert errs[0] < 6e-3
    assert errs[1] < 0.5 * errs[0]          # first order at the shocks at least


def test_sod_1024_known_answer():
    q, r, e = sod(1024)
    rho = q[0, 0, :, 0]
    u = q[0, 0, :, 1] / rho
    assert np.mean(np.abs(rho - e[0])) < 1.5e-3
    assert np.mean(np.abs(u - e[1])) < 3e-3
    assert r["steps"] > 200


@pytest.mark.parametrize("solver", [1, 2])
@pytest.mark.parametrize("limiter", [1, 2, 3])
def test_periodic_conservation(solver, limiter):
    o = Oracle(make_params(nx=12, ny=10, nz=8, boundtype=2, solver=solver, limiter=limiter, g=5 / 3, cfl=0.3))
    q = random_q(o, np.random.default_rng(3), rho=(0.8, 1.2), vel=(-0.2, 0.2), pres=(0.8, 1.2))
    tot0 = q.reshape(-1, 6).sum(0)
    for _ in range(5):
        q, dt, t = oracle_step(o, q)
    assert o.error() == 0
    tot = q.reshape(-1, 6).sum(0)
    scale = np.abs(q.reshape(-1, 6)).sum(0)
    assert np.all(np.abs(tot[:5] - tot0[:5]) <= 1e-13 * scale[:5])


def test_shocktube_direction_symmetry():
    profiles = []
    for d in (1, 2, 3):
        n = [4, 4, 4]
        n[d - 1] = 64
        o = Oracle(make_params(nx=n[0], ny=n[1], nz=n[2], g=1.4, cfl=0.8, boundtype=1, tend=0.05))
        q = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, d)
        r = o.run(q, 1000)
        assert r["status"] == 0
        prof = np.moveaxis(q, (2, 1, 0)[d - 1], 0)[:, 0, 0, :].copy()
        # the momentum along d moves into field 1
        prof[:, [1, d]] = prof[:, [d, 1]]
        profiles.append((r["steps"], prof))
    assert profiles[0][0] == profiles[1][0] == profiles[2][0]
    np.testing.assert_array_equal(profiles[0][1], profiles[1][1])
    np.testing.assert_array_equal(profiles[0][1], profiles[2][1])


def test_negative_pressure_is_reported():
    o = Oracle(make_params(nx=16, ny=1, nz=1, boundtype=1))
    q = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1)
    q[0, 0, 5, 4] = 0.0              # E = 0 -> p <= 0
    r = o.run(q, 1)
    assert r["status"] & 1


def test_hllc_matches_hll_on_a_contact_free_state():
    o = Oracle(make_params(nx=8, ny=1, nz=1, g=1.4))
    wl = np.array([1.0, 0.3, 0.0, 0.0, 1.0])
    f_hllc = o.riemann(wl, wl, 1)
    o2 = Oracle(make_params(nx=8, ny=1, nz=1, g=1.4, solver=1))
    f_hll = o2.riemann(wl, wl, 1)
    # identical states: both return the physical flux
    np.testing.assert_allclose(f_hllc, f_hll, rtol=1e-15)
    assert f_hllc[0] == pytest.approx(0.3)


def test_parameter_defaults_follow_readparameter():
    p = make_params()
    o = Oracle(p)
    assert o.d.g == float(np.float32(1.4))          # default-real literal
    o.configure(make_params(atomic=1, g=1.4))
    assert o.d.g == float(np.float32(5.0) / np.float32(3.0))
    o.configure(make_params(nx=64, ny=1, nz=1))
    assert o.d.dy == o.d.dx and o.d.dz == o.d.dx   # parameter.f90:195-205
