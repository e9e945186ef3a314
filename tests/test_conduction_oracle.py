"""Thermal conduction (conduction.f90, thermalstep timestep.f90:72-104) in
the hand-written oracle against the reference's own Fortran translated to C
(oracle/_ref): bit for bit, routine by routine and over runs with the hydro
steps (main.f90:121, 169-175).  Only the simplekappa branch is defined in
the reference's plain build; the other branch is refused."""
import numpy as np
import pytest

from oracle import ref_oracle
from oracle.oracle import Oracle, make_params
from oracle.ref_oracle import RefOracle
from helpers import random_q

pytestmark = pytest.mark.skipif(not ref_oracle.available(), reason="translated reference not built")

# boxes large enough that the explicit conduction (kappa_eff = 1/(g-1)) is
# stable at the hydro CFL step
CONFIGS = [
    dict(nx=13, ny=11, nz=9, boundtype=2, xmax=52.0, ymax=44.0, zmax=36.0),
    dict(nx=13, ny=11, nz=9, boundtype=1, xmax=52.0, ymax=44.0, zmax=36.0, limiter=2),
    dict(nx=24, ny=17, nz=1, boundtype=3, xmax=96.0, ymax=68.0),
    dict(nx=64, ny=1, nz=1, boundtype=1, xmax=256.0),
    dict(nx=12, ny=10, nz=8, boundtype=2, xmax=48.0, ymax=40.0, zmax=32.0, dualenergy=1, de_thresh=0.3),
]


def params(cfg):
    return make_params(g=5 / 3, cfl=0.4, conduction=1, simplekappa=1, tend=1e6, **cfg)


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_conduction_routines_match_reference_bitwise(cfg):
    o, r = Oracle(params(cfg)), RefOracle(params(cfg))
    q = random_q(o, np.random.default_rng(5), pres=(0.5, 3.0))
    if cfg.get("dualenergy"):
        q[..., 5] *= 1.02
    w = np.zeros(o.shape_w)
    q_o, q_r = q.copy(), q.copy()
    o.primitive(w, q_o)
    r.primitive(w.copy(), q_r)
    o.bound(w)
    w_r = w.copy()
    dt_o = o.thermalstep(q_o, w, 0.7)
    dt_r, st = r.thermalstep(q_r, w_r, 0.7)
    assert st == 0 and dt_o == dt_r
    np.testing.assert_array_equal(q_o, q_r)
    assert o.thermalstep(q_o.copy(), w, 1e99) < 1e99    # the limit itself is finite
    o.thermalconduction(q_o, w, 0.37)
    assert r.thermalconduction(q_r, w_r, 0.37) == 0
    np.testing.assert_array_equal(q_o, q_r)
    assert not np.array_equal(q_o[..., 4], q[..., 4])


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_runs_with_conduction_match_reference_bitwise(cfg):
    o, r = Oracle(params(cfg)), RefOracle(params(cfg))
    q = random_q(o, np.random.default_rng(6), pres=(0.5, 3.0))
    q_o, q_r = q.copy(), q.copy()
    a = o.run(q_o, 12)
    b = r.run(q_r, 12)
    assert a["status"] == 0 and b["stopped"] == 0 and a["steps"] == b["steps"] == 12
    assert a["t"] == b["t"] and a["dt"] == b["dt"]
    np.testing.assert_array_equal(q_o, q_r)


def test_non_simplekappa_is_refused():
    with pytest.raises(ValueError):
        Oracle(make_params(nx=8, ny=8, nz=8, conduction=1, simplekappa=0))
