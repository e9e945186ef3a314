"""The plain-build chem(q) step (pressure floors, chemistry.f90:72-121) on
the GPU against the oracle, which is pinned bit for bit to the reference's
translated Fortran: the drop-in routine and grids that apply the floors
after every hydro step.  E bit-exact in strict FP64; S through the device
pow."""
import numpy as np
import pytest

import evora_b200 as ev
from helpers import random_q
from oracle.oracle import Oracle, make_params

pytestmark = pytest.mark.gpu

CASES = [
    dict(nx=13, ny=11, nz=9, boundtype=2, tempfloor=1, temp_fl=1.2),
    dict(nx=24, ny=17, nz=1, boundtype=3, tempfloor=1, temp_fl=0.9, jeansfloor=1, c_jeans=0.05),
    dict(nx=64, ny=1, nz=1, boundtype=1, jeansfloor=1, c_jeans=0.01, fb=0.8),
    dict(nx=12, ny=10, nz=8, boundtype=2, dualenergy=1, de_thresh=0.3, tempfloor=1, temp_fl=1.1),
]
IDS = ["3d-temp", "2d-both", "1d-jeans", "3d-dual-energy"]


def kw_of(cfg):
    return dict(g=5 / 3, cfl=0.4, tend=1e6, **cfg)


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_dropin_chem_matches_oracle(cuda_device, cfg):
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(14), pres=(0.3, 3.0))
    if cfg.get("dualenergy"):
        q[..., 5] *= 1.02
    q_o, q_g = q.copy(), q.copy()
    o.chem(q_o)
    ev.DropIn(ev.default_params(**kw), strict=True).chem(q_g)
    np.testing.assert_array_equal(q_g[..., :5], q_o[..., :5])
    np.testing.assert_allclose(q_g[..., 5], q_o[..., 5], rtol=1e-14)


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_grid_with_floors_matches_oracle(cuda_device, cfg):
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(15), pres=(0.3, 3.0))
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


def test_fp32_floors_close_to_fp64(cuda_device):
    kw = kw_of(CASES[0])
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(16), pres=(0.3, 3.0))
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(ev.default_params(**kw), prec) as g:
            g.set_q(q0)
            g.step(10)
            out[prec] = g.get_q()
    for f in (0, 4):
        a, b = out[ev.FP32][..., f], out[ev.FP64][..., f]
        assert np.abs(a - b).sum() / np.abs(b).sum() < 1e-5
