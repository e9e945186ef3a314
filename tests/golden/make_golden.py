"""Generates the golden fixtures of tests/golden/ from the reference's own
hydro path (its Fortran sources translated mechanically to C by
oracle/ref/f2c.py and driven like main.f90 by oracle/ref/harness.c).

Run from the repository root where /root/reference exists:
    python tests/golden/make_golden.py [classic] [conduction]
Each fixture holds the inputs (parameters, initial q) and the reference's
outputs (q after the steps, t, dt, steps).  The reference itself has no test
vectors (its bin/test only draws plots)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.oracle import make_params  # noqa: E402
from oracle.ref_oracle import RefOracle  # noqa: E402
from helpers import random_q  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["nx", "ny", "nz", "solver", "limiter", "boundtype", "secondorder", "dualenergy", "atomic",
          "g", "cfl", "de_thresh", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "tstart", "tend",
          "conduction", "simplekappa", "c_cond"]


class _O:
    """Minimal stand-in for helpers.random_q (needs .p, .d.g1, zeros_q)."""

    def __init__(self, r):
        self.p = r.p
        self.d = type("D", (), {"g1": r.derived["g1"]})
        self.zeros_q = r.zeros_q


def save(name, kw, q0, steps):
    r = RefOracle(make_params(**kw))
    q = q0.copy()
    res = r.run(q, steps)
    assert res["stopped"] == 0, name
    p = make_params(**kw)
    np.savez_compressed(os.path.join(HERE, name + ".npz"),
                        params=np.array([getattr(p, f) for f in FIELDS], dtype=np.float64),
                        q0=q0, q=q, t=res["t"], dt=res["dt"], steps=res["steps"], go=res["go"])
    print(name, res)


def main(only=None):
    if only:
        # a subset by name (the other fixtures stay as committed)
        for name in only:
            CASES[name]()
        return
    for make in CASES.values():
        make()


def _conduction():
    # thermal conduction (simplekappa) after every hydro step, 3D, a box
    # large enough for the explicit conduction to be stable
    kw = dict(nx=14, ny=12, nz=10, g=5 / 3, cfl=0.4, boundtype=1, limiter=1, tend=100.0,
              xmax=56.0, ymax=48.0, zmax=40.0, conduction=1, simplekappa=1)
    r = RefOracle(make_params(**kw))
    save("cond3d_14x12x10_simplekappa", kw, random_q(_O(r), np.random.default_rng(11), pres=(0.5, 3.0)), 8)


def _classic():
    kw = dict(nx=1024, ny=1, nz=1, g=1.4, cfl=0.8, boundtype=1, tend=0.2)
    r = RefOracle(make_params(**kw))
    save("sod1024_hllc_minmod", kw, r.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1), 100000)

    kw = dict(nx=512, ny=1, nz=1, g=1.4, cfl=0.5, boundtype=3, tend=0.15, solver=1, limiter=3)
    r = RefOracle(make_params(**kw))
    save("sod512_hll_vanleer_reflect", kw, r.ic_shocktube(1.0, 0.75, 1.0, 0.125, 0.0, 0.1, 0.3, 1), 100000)

    kw = dict(nx=32, ny=32, nz=1, cfl=0.5, boundtype=2, limiter=2, tend=100.0)   # para/kevinhelmholtz
    r = RefOracle(make_params(**kw))
    save("kh2d_32_moncen", kw, r.ic_kh2d(), 20)

    kw = dict(nx=16, ny=12, nz=8, g=5 / 3, cfl=0.4, boundtype=3, limiter=2, solver=1, tend=100.0)
    r = RefOracle(make_params(**kw))
    save("random3d_hll_moncen_bt3", kw, random_q(_O(r), np.random.default_rng(7)), 4)

    kw = dict(nx=16, ny=12, nz=10, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    r = RefOracle(make_params(**kw))
    from evora_b200 import ic, default_params
    save("kh3d_16x12x10", kw, ic.kh3d(default_params(**kw)), 10)


CASES = {"classic": _classic, "conduction": _conduction}

if __name__ == "__main__":
    main(sys.argv[1:] or None)
