"""The drop-in routines in resident mode (evora_set_resident): main.f90's
call order (primitive, bound, hydrostep, updatetime, compevo, sweep;
main.f90:109-155) with host arrays, the state kept on the GPU between calls
and brought back by evora_sync.  Against the oracle's time loop on the same
inputs: strict FP64 bit-exact on rho, m, E with the same times over 10
steps; default FP64 within 1e-12 relative L1; the FP32 form within 1e-5 in
density.  Host q stays as it was until synced; a routine that changes q on
the host (chem) in between makes the next primitive upload it again."""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import random_q, rel_l1

pytestmark = pytest.mark.gpu

CONFIGS = [
    dict(nx=32, ny=16, nz=12, boundtype=2),                 # whole tiles: the staged kernels
    dict(nx=13, ny=11, nz=9, boundtype=1, limiter=2),
    dict(nx=20, ny=14, nz=10, boundtype=3, solver=1),
    dict(nx=24, ny=17, nz=1, boundtype=3),
    dict(nx=300, ny=1, nz=1, boundtype=1),
]


def main_loop(di, p, q, steps):
    """main.f90:109-155 through the drop-in routines on host arrays."""
    sh = ev.shapes(p)
    w, evo, s = np.zeros(sh["w"]), np.zeros(sh["evo"]), np.zeros(sh["s"])
    t, go, k = p.tstart, True, 0
    while go and k < steps:
        di.primitive(w, q)
        di.bound(w)
        dt = di.hydrostep(w, 1e99)
        go, t, dt = di.updatetime(go, t, dt)
        if p.secondorder:
            di.compevo(w, evo, s, dt)
        di.sweep(w, q, evo, s, dt)
        k += 1
    return t, k, (w, evo, s)


def oracle_run(kw, q, steps):
    o = Oracle(make_params(**kw))
    qo = q.copy()
    r = o.run(qo, steps)
    assert r["status"] == 0
    return qo, r


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_resident_strict_matches_oracle_bitwise(cuda_device, cfg):
    kw = dict(g=5 / 3, cfl=0.4, tend=10.0, **cfg)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(3), rho=(0.8, 1.2), vel=(-0.2, 0.2), pres=(0.8, 1.2))
    qo, r = oracle_run(kw, q0, 10)
    p = ev.default_params(**kw)
    di = ev.DropIn(p, strict=True)
    di.set_resident(ev.RESIDENT_FP64)
    try:
        q = q0.copy()
        t, k, (w, evo, s) = main_loop(di, p, q, 10)
        np.testing.assert_array_equal(q, q0)      # host q is untouched until synced
        assert not w.any() and not evo.any() and not s.any()   # w, evo, s are never written
        di.sync(q)
    finally:
        di.set_resident(0)
    assert k == r["steps"] and t == r["t"]
    np.testing.assert_array_equal(q[..., :5], qo[..., :5])


@pytest.mark.parametrize("mode, tol", [(ev.RESIDENT_FP64, 1e-12), (ev.RESIDENT_FP32, 1e-5)], ids=["fp64", "fp32"])
def test_resident_default_forms(cuda_device, mode, tol):
    kw = dict(nx=64, ny=32, nz=24, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    p = ev.default_params(**kw)
    q0 = ev.ic.kh3d(p)
    qo, r = oracle_run(kw, q0, 10)
    di = ev.DropIn(p)
    di.set_resident(mode)
    try:
        q = q0.copy()
        t, k, _ = main_loop(di, p, q, 10)
        di.sync(q)
    finally:
        di.set_resident(0)
    assert k == 10 and abs(t - r["t"]) <= 1e-6 * r["t"]
    err = rel_l1(q[..., :5], qo[..., :5])
    assert err[0] <= tol, err
    if mode == ev.RESIDENT_FP64:
        assert np.all(err[[0, 1, 2, 4]] <= tol), err


def test_resident_host_changes_are_uploaded(cuda_device):
    # the plain build's chem(q) (the temperature floor) between steps: the
    # state goes to the host first, chem runs there, the next primitive
    # uploads the changed q; equal to the same loop without residency
    kw = dict(nx=16, ny=16, nz=8, g=5 / 3, cfl=0.4, boundtype=2, tend=10.0, tempfloor=1, temp_fl=3e4)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(5), pres=(0.05, 2.0))
    p = ev.default_params(**kw)
    outs = []
    for resident in (0, ev.RESIDENT_FP64):
        di = ev.DropIn(p, strict=True)
        di.set_resident(resident)
        q = q0.copy()
        for _ in range(3):
            main_loop(di, p, q, 1)
            di.chem(q)
        di.sync(q)
        di.set_resident(0)
        outs.append(q)
    assert not np.array_equal(outs[0], q0)
    np.testing.assert_array_equal(outs[1][..., :5], outs[0][..., :5])


def test_resident_errors(cuda_device):
    p = ev.default_params(nx=16, ny=8, nz=8, g=5 / 3, boundtype=2)
    di = ev.DropIn(p)
    di.set_resident(ev.RESIDENT_FP64)
    try:
        sh = ev.shapes(p)
        w = np.zeros(sh["w"])
        with pytest.raises(ev.EvoraError):
            di.hydrostep(w)                       # nothing bound yet
        q = ev.ic.kh3d(p)
        q[2, 3, 4, 4] = -1.0                      # negative energy: p <= 0
        di.primitive(w, q)
        with pytest.raises(ev.EvoraError) as e:
            di.hydrostep(w)
        assert e.value.status & 1
    finally:
        di.set_resident(0)
    with pytest.raises(ev.EvoraError):
        di.set_resident(7)
