"""The oracle pinned to the reference's own sources.

oracle/_ref is the reference's Fortran hydro path (global.f90,
compparameter, decomposition, comp.f90, muscl.f90, riemann.f90, boundary.f90,
hydrostep, updatetime, ic/shocktube.f90, ic/kevinhelmholtz.f90) translated
mechanically to C (oracle/ref/f2c.py) and driven like main.f90.  The
hand-written oracle must reproduce it bit for bit, routine by routine and
over full runs; both must reproduce the golden fixtures of tests/golden/
(made from oracle/_ref by tests/golden/make_golden.py)."""
import glob
import os

import numpy as np
import pytest

from oracle import ref_oracle
from oracle.oracle import Oracle, make_params
from oracle.ref_oracle import RefOracle
from helpers import random_q

pytestmark = pytest.mark.skipif(not ref_oracle.available(), reason="translated reference not built")

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
FIELDS = ["nx", "ny", "nz", "solver", "limiter", "boundtype", "secondorder", "dualenergy", "atomic",
          "g", "cfl", "de_thresh", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "tstart", "tend",
          "conduction", "simplekappa", "c_cond"]
INT_FIELDS = set(FIELDS[:9]) | {"conduction", "simplekappa"}


def params_of(arr):
    kw = {}
    for f, v in zip(FIELDS, arr):
        kw[f] = int(v) if f in INT_FIELDS else float(v)
    return kw


CONFIGS = [
    dict(nx=13, ny=11, nz=9, boundtype=2),
    dict(nx=13, ny=11, nz=9, boundtype=1, limiter=2),
    dict(nx=13, ny=11, nz=9, boundtype=3, limiter=3, solver=1),
    dict(nx=24, ny=17, nz=1, boundtype=3, limiter=2),
    dict(nx=24, ny=17, nz=1, boundtype=1, solver=1),
    dict(nx=64, ny=1, nz=1, boundtype=1),
    dict(nx=40, ny=1, nz=1, boundtype=3, limiter=3),
    dict(nx=13, ny=11, nz=9, boundtype=2, secondorder=0),
    dict(nx=12, ny=10, nz=8, boundtype=2, dualenergy=1, de_thresh=0.3),
    dict(nx=12, ny=10, nz=8, boundtype=1, atomic=1),
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_routines_match_reference_bitwise(cfg):
    kw = dict(g=5 / 3, cfl=0.4, **cfg)
    o = Oracle(make_params(**kw))
    r = RefOracle(make_params(**kw))
    for k, v in r.derived.items():
        assert getattr(o.d, k) == v, k
    q = random_q(o, np.random.default_rng(3), vel=(-1.0, 1.0))
    if cfg.get("dualenergy"):
        q[..., 5] *= 1.02
    rng = np.random.default_rng(4)
    w_o = rng.uniform(1, 2, o.shape_w)
    w_r = w_o.copy()
    q_o, q_r = q.copy(), q.copy()
    o.primitive(w_o, q_o)
    assert r.primitive(w_r, q_r) == 0
    np.testing.assert_array_equal(w_o, w_r)
    np.testing.assert_array_equal(q_o, q_r)          # dual-energy write-back
    o.bound(w_o)
    r.bound(w_r)
    np.testing.assert_array_equal(w_o, w_r)
    dt_o = o.hydrostep(w_o, 1e99)
    dt_r, st = r.hydrostep(w_r, 1e99)
    assert st == 0 and dt_o == dt_r
    assert o.updatetime(0.0, dt_o) == r.updatetime(0.0, dt_r)
    evo_o, s_o = np.zeros(o.shape_evo), np.zeros(o.shape_s)
    evo_r, s_r = np.zeros(o.shape_evo), np.zeros(o.shape_s)
    o.compevo(w_o, evo_o, s_o, dt_o)
    r.compevo(w_r, evo_r, s_r, dt_r)
    np.testing.assert_array_equal(s_o, s_r)
    np.testing.assert_array_equal(evo_o, evo_r)
    o.sweep(w_o, q_o, evo_o, s_o, dt_o)
    assert r.sweep(w_r, q_r, evo_r, s_r, dt_r) == 0
    np.testing.assert_array_equal(q_o, q_r)
    assert o.error() == 0


@pytest.mark.parametrize("direction", [1, 2, 3])
def test_shocktube_ic_and_run_match_reference(direction):
    n = [6, 5, 4]
    n[direction - 1] = 48
    kw = dict(nx=n[0], ny=n[1], nz=n[2], g=1.4, cfl=0.4, boundtype=3, tend=0.05)
    o, r = Oracle(make_params(**kw)), RefOracle(make_params(**kw))
    args = (1.0, 0.3, 1.0, 0.125, -0.2, 0.1, 0.45, direction)
    qo, qr = o.ic_shocktube(*args), r.ic_shocktube(*args)
    np.testing.assert_array_equal(qo, qr)
    ro, rr = o.run(qo, 1000), r.run(qr, 1000)
    assert (ro["steps"], ro["t"], ro["dt"]) == (rr["steps"], rr["t"], rr["dt"])
    np.testing.assert_array_equal(qo, qr)


def test_kh2d_ic_matches_reference():
    kw = dict(nx=40, ny=40, nz=1)
    np.testing.assert_array_equal(Oracle(make_params(**kw)).ic_kh2d(), RefOracle(make_params(**kw)).ic_kh2d())


def test_riemann_solvers_match_reference():
    rng = np.random.default_rng(9)
    for solver in (1, 2):
        o = Oracle(make_params(nx=8, ny=1, nz=1, g=5 / 3, solver=solver))
        r = RefOracle(make_params(nx=8, ny=1, nz=1, g=5 / 3, solver=solver))
        for _ in range(500):
            wl = np.r_[rng.uniform(0.1, 10), rng.uniform(-3, 3, 3), rng.uniform(0.01, 10)]
            wr = np.r_[rng.uniform(0.1, 10), rng.uniform(-3, 3, 3), rng.uniform(0.01, 10)]
            d = int(rng.integers(1, 4))
            fr, st = r.riemann(wl, wr, d)
            assert st == 0
            np.testing.assert_array_equal(o.riemann(wl, wr, d), fr)


def test_negative_pressure_stops_both():
    kw = dict(nx=16, ny=1, nz=1, boundtype=1)
    o, r = Oracle(make_params(**kw)), RefOracle(make_params(**kw))
    q = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1)
    q[0, 0, 5, 4] = 0.0
    assert o.run(q.copy(), 1)["status"] & 1
    assert r.run(q.copy(), 1)["stopped"] == 1


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_golden_fixtures(path):
    g = np.load(path)
    kw = params_of(g["params"])
    for make in (Oracle, RefOracle):
        o = make(make_params(**kw))
        q = g["q0"].copy()
        res = o.run(q, int(g["steps"]))
        assert res["steps"] == int(g["steps"]) and res["t"] == float(g["t"]) and res["dt"] == float(g["dt"])
        np.testing.assert_array_equal(q, g["q"])
