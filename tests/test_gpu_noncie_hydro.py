"""The non-equilibrium build's hydro path on the GPU (the reference compiled
with -DNONCIE: q(12) with all 12 fields advected, w(11) with the species per
unit mass, global.f90:30-36): the drop-in routines primitive, bound,
hydrostep, compevo and sweep against the reference's own Fortran translated
with -DNONCIE (oracle/_ref/libevora_ref_ncie.so), routine by routine bit for
bit in strict FP64 (the species rows of flux, state and statex,
riemann.f90:200-204, 233-237, 282-286; the species slopes and predictor,
muscl.f90:62-111; integration over nf = 12, muscl.f90:284-285), and over a
20-step comoving run with the Patankar chem(q) after every sweep
(main.f90:109-167) to the tolerance of the device's exp and log."""
import numpy as np
import pytest

import evora_b200 as ev
from helpers import random_q
from oracle.oracle import Oracle, make_params
from oracle.ref_oracle import RefOracle

pytestmark = pytest.mark.gpu

HYDRO = [
    dict(nx=12, ny=10, nz=8, boundtype=2),
    dict(nx=11, ny=9, nz=7, boundtype=3, limiter=2, solver=1),
    dict(nx=20, ny=13, nz=1, boundtype=1, limiter=3),
    dict(nx=48, ny=1, nz=1, boundtype=3),
]


def ncie_state(kw, seed):
    """A random flow with the species of initchem scaled by random factors,
    so that every species varies between cells."""
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(seed), rho=(0.5, 2.0), pres=(0.5, 2.0))
    o.initchem(q)
    rng = np.random.default_rng(seed + 1)
    q[..., 6:] = np.maximum(q[..., 6:], 1e-3 * q[..., :1]) * rng.uniform(0.5, 1.5, q[..., 6:].shape)
    return q


@pytest.mark.parametrize("cfg", HYDRO, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_noncie_dropin_routines_bitwise(cuda_device, cfg):
    kw = dict(chemistry=1, noncie=1, g=5 / 3, cfl=0.4, **cfg)
    q0 = ncie_state(kw, 3)
    ref = RefOracle(make_params(**kw))
    di = ev.DropIn(ev.default_params(**kw), strict=True)
    assert ref.shape_w[-1] == 11 and di.shape["w"][-1] == 11
    w_r, w_g = np.zeros(ref.shape_w), np.zeros(ref.shape_w)
    q_r, q_g = q0.copy(), q0.copy()
    assert ref.primitive(w_r, q_r) == 0
    di.primitive(w_g, q_g)
    assert ref.bound(w_r) == 0
    di.bound(w_g)
    np.testing.assert_array_equal(w_g, w_r)
    dt_r, st = ref.hydrostep(w_r)
    assert st == 0 and di.hydrostep(w_g) == dt_r
    e_r, e_g = np.zeros(ref.shape_evo), np.zeros(ref.shape_evo)
    s_r, s_g = np.zeros(ref.shape_s), np.zeros(ref.shape_s)
    assert ref.compevo(w_r, e_r, s_r, dt_r) == 0
    di.compevo(w_g, e_g, s_g, dt_r)
    np.testing.assert_array_equal(s_g, s_r)
    np.testing.assert_array_equal(e_g, e_r)
    assert ref.sweep(w_r, q_r, e_r, s_r, dt_r) == 0
    di.sweep(w_g, q_g, e_g, s_g, dt_r)
    # the entropy row goes through pow (device vs libm); every other field,
    # the species included, is bit for bit
    keep = [f for f in range(12) if f != 5]
    np.testing.assert_array_equal(q_g[..., keep], q_r[..., keep])
    np.testing.assert_allclose(q_g[..., 5], q_r[..., 5], rtol=1e-13)
    assert not np.array_equal(q_r[..., 6:], q0[..., 6:])   # the species moved


def test_noncie_run_with_chemistry(cuda_device):
    kw = dict(chemistry=1, noncie=1, cooling=1, atomic=1, supercomoving=1, omega0=0.3, lambda0=0.7,
              hubble0=70.0, box=1.0, zstart=10.0, zend=9.0, g=5 / 3, cfl=0.4, nx=12, ny=10, nz=8,
              boundtype=2)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(9), rho=(0.5, 2.0), vel=(-0.05, 0.05), pres=(0.5, 2.0))
    o.initchem(q0)
    ref = RefOracle(make_params(**kw))
    q_r = q0.copy()
    r = ref.run(q_r, 20)
    assert r["stopped"] == 0 and r["steps"] == 20
    di = ev.DropIn(ev.default_params(**kw), strict=True)
    sh = di.shape
    w, evo, s = np.zeros(sh["w"]), np.zeros(sh["evo"]), np.zeros(sh["s"])
    q = q0.copy()
    ts = di.cosmostart()
    go, k4 = True, 1
    for _ in range(20):
        di.primitive(w, q)
        di.bound(w)
        ts["dt"] = di.hydrostep(w, 1e99)
        ts = di.compcosmo(di.cosmostep(ts))
        go, dump, ts = di.updatetime_cosmo(go, ts, k4)
        di.settime(ts)
        di.compevo(w, evo, s, ts["dt"])
        di.sweep(w, q, evo, s, ts["dt"])
        di.chem(q)
        if dump:
            k4 += 1
    assert ts["t"] == r["t"]
    rel = np.abs(q - q_r) / np.maximum(np.abs(q_r), 1e-300)
    assert rel[..., :5].max() < 1e-9, rel[..., :5].max()
    assert rel[..., 6:].max() < 1e-8, rel[..., 6:].max()
