"""Thermal conduction on the GPU (conduction.f90, thermalstep
timestep.f90:72-104, simplekappa) against the oracle, whose conduction is
pinned bit for bit to the reference's translated Fortran: the drop-in
routines on the reference layouts and grids that conduct after every hydro
step.  E is bit-exact in strict FP64; S goes through the device pow."""
import numpy as np
import pytest

import evora_b200 as ev
from helpers import random_q
from oracle.oracle import Oracle, make_params

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx=13, ny=11, nz=9, boundtype=2, xmax=52.0, ymax=44.0, zmax=36.0),
    dict(nx=24, ny=17, nz=1, boundtype=3, xmax=96.0, ymax=68.0),
    dict(nx=64, ny=1, nz=1, boundtype=1, xmax=256.0),
    dict(nx=12, ny=10, nz=8, boundtype=1, xmax=48.0, ymax=40.0, zmax=32.0, dualenergy=1, de_thresh=0.3),
]
IDS = ["3d-periodic", "2d-reflect", "1d", "3d-dual-energy"]


def kw_of(cfg):
    return dict(g=5 / 3, cfl=0.4, conduction=1, simplekappa=1, tend=1e6, **cfg)


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_dropin_conduction_matches_oracle(cuda_device, cfg):
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    d = ev.DropIn(ev.default_params(**kw), strict=True)
    q = random_q(o, np.random.default_rng(8), pres=(0.5, 3.0))
    if cfg.get("dualenergy"):
        q[..., 5] *= 1.02
    w = np.zeros(o.shape_w)
    o.primitive(w, q)
    o.bound(w)
    q_o, q_g = q.copy(), q.copy()
    dt_o = o.thermalstep(q_o, w, 1e99)
    dt_g = d.thermalstep(q_g, w, 1e99)
    assert dt_g == pytest.approx(dt_o, rel=1e-14)     # T^2.5 through the device pow
    np.testing.assert_allclose(q_g, q_o, rtol=1e-15, atol=0)
    q_o, q_g = q.copy(), q.copy()
    o.thermalconduction(q_o, w, 0.31)
    d.thermalconduction(q_g, w, 0.31)
    np.testing.assert_array_equal(q_g[..., :5], q_o[..., :5])
    np.testing.assert_allclose(q_g[..., 5], q_o[..., 5], rtol=1e-14)


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_grid_with_conduction_matches_oracle(cuda_device, cfg):
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(9), pres=(0.5, 3.0))
    q_o = q0.copy()
    res = o.run(q_o, 10)
    assert res["status"] == 0
    with ev.Grid(ev.default_params(**kw), ev.FP64, ev.STRICT | ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        g.step(10)
        t = g.time()
        q = g.get_q()
    assert t["k"] == 10 and t["t"] == res["t"] and t["dt"] == res["dt"]
    np.testing.assert_array_equal(q[..., :5], q_o[..., :5])
    np.testing.assert_allclose(q[..., 5], q_o[..., 5], rtol=1e-13)


def test_fp32_conduction_close_to_fp64(cuda_device):
    kw = kw_of(CASES[0])
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(10), pres=(0.5, 3.0))
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(ev.default_params(**kw), prec) as g:
            g.set_q(q0)
            g.step(10)
            out[prec] = g.get_q()
    for f in (0, 4):
        a, b = out[ev.FP32][..., f], out[ev.FP64][..., f]
        assert np.abs(a - b).sum() / np.abs(b).sum() < 1e-5


def test_spitzer_branch_is_refused(cuda_device):
    with pytest.raises(ev.EvoraError):
        ev.Grid(ev.default_params(nx=8, ny=8, nz=8, conduction=1, simplekappa=0), ev.FP64)
