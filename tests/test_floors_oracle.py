"""chem(q) of the reference's plain build (chemistry.f90:72-121: pressure()
and the temperature / Jeans pressure floors, main.f90:167) in the hand
oracle against the reference's Fortran translated to C: bit for bit for the
routine and for runs with the hydro steps."""
import numpy as np
import pytest

from oracle import ref_oracle
from oracle.oracle import Oracle, make_params
from oracle.ref_oracle import RefOracle
from helpers import random_q

pytestmark = pytest.mark.skipif(not ref_oracle.available(), reason="translated reference not built")

CONFIGS = [
    dict(nx=13, ny=11, nz=9, boundtype=2, tempfloor=1, temp_fl=1.2),
    dict(nx=13, ny=11, nz=9, boundtype=1, jeansfloor=1, c_jeans=0.01, fb=0.8),
    dict(nx=24, ny=17, nz=1, boundtype=3, tempfloor=1, temp_fl=0.9, jeansfloor=1, c_jeans=0.05),
    dict(nx=64, ny=1, nz=1, boundtype=1, tempfloor=1, temp_fl=1.5),
    dict(nx=12, ny=10, nz=8, boundtype=2, dualenergy=1, de_thresh=0.3, tempfloor=1, temp_fl=1.1),
]


def params(cfg):
    return make_params(g=5 / 3, cfl=0.4, tend=1e6, **cfg)


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_chem_floors_match_reference_bitwise(cfg):
    o, r = Oracle(params(cfg)), RefOracle(params(cfg))
    q = random_q(o, np.random.default_rng(12), pres=(0.3, 3.0))
    if cfg.get("dualenergy"):
        q[..., 5] *= 1.02
    q_o, q_r = q.copy(), q.copy()
    o.chem(q_o)
    assert r.chem(q_r) == 0
    np.testing.assert_array_equal(q_o, q_r)
    assert not np.array_equal(q_o[..., 4], q[..., 4])      # some floor acted


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_runs_with_floors_match_reference_bitwise(cfg):
    o, r = Oracle(params(cfg)), RefOracle(params(cfg))
    q = random_q(o, np.random.default_rng(13), pres=(0.3, 3.0))
    q_o, q_r = q.copy(), q.copy()
    a = o.run(q_o, 10)
    b = r.run(q_r, 10)
    assert a["status"] == 0 and b["stopped"] == 0 and a["steps"] == b["steps"] == 10
    assert a["t"] == b["t"] and a["dt"] == b["dt"]
    np.testing.assert_array_equal(q_o, q_r)
