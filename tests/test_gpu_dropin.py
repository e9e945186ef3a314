"""Drop-in routines (primitive, bound, hydrostep, updatetime, compevo, sweep)
on the GPU against the oracle's restatement of the same subroutines, called
through the C ABI on the same inputs.  Strict mode (no FMA contraction) must
be bit-exact on rho, m, E and all of w, s, evo; the entropy field S goes
through pow (device vs glibc) and is compared to 1e-14.  The default mode is
compared to 1e-12 relative."""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import random_q

pytestmark = pytest.mark.gpu

CONFIGS = [
    dict(nx=13, ny=11, nz=9, boundtype=2),
    dict(nx=13, ny=11, nz=9, boundtype=1, limiter=2),
    dict(nx=13, ny=11, nz=9, boundtype=3, limiter=3, solver=1),
    dict(nx=24, ny=17, nz=1, boundtype=3),
    dict(nx=64, ny=1, nz=1, boundtype=1),
    dict(nx=40, ny=1, nz=1, boundtype=3, solver=1, secondorder=0),
]


def setup(cfg, seed=0):
    kw = dict(g=5 / 3, cfl=0.4, **cfg)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(seed))
    return o, ev.default_params(**kw), q


def assert_match(a, b, strict, what):
    if strict:
        np.testing.assert_array_equal(a, b, err_msg=what)
    else:
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-13, err_msg=what)


@pytest.mark.parametrize("strict", [True, False])
@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_dropin_step_matches_oracle(cuda_device, cfg, strict):
    o, p, q = setup(cfg)
    di = ev.DropIn(p, strict=strict)
    sh = ev.shapes(p)
    rng = np.random.default_rng(1)
    # ghost cells start with junk: bound must overwrite exactly what the reference does
    w_o = rng.uniform(1, 2, sh["w"])
    w_g = w_o.copy()
    o.primitive(w_o, q.copy())
    di.primitive(w_g, q.copy())
    assert_match(w_g, w_o, strict, "primitive")
    o.bound(w_o)
    di.bound(w_g)
    assert_match(w_g, w_o, strict, "bound")
    w_g = w_o.copy()
    dt_o = o.hydrostep(w_o, 1e99)
    dt_g = di.hydrostep(w_g, 1e99)
    assert dt_g == dt_o
    go_o, t_o, dt_o2 = o.updatetime(0.0, dt_o)
    go_g, t_g, dt_g2 = di.updatetime(True, 0.0, dt_g)
    assert (go_o, t_o, dt_o2) == (go_g, t_g, dt_g2)
    evo_o, s_o = np.zeros(sh["evo"]), np.zeros(sh["s"])
    evo_g, s_g = np.zeros(sh["evo"]), np.zeros(sh["s"])
    if p.secondorder:
        o.compevo(w_o, evo_o, s_o, dt_o2)
        di.compevo(w_g, evo_g, s_g, dt_g2)
        assert_match(s_g, s_o, strict, "slopes")
        assert_match(evo_g, evo_o, strict, "evo")
    q_o, q_g = q.copy(), q.copy()
    o.sweep(w_o, q_o, evo_o, s_o, dt_o2)
    di.sweep(w_o, q_g, evo_o, s_o, dt_o2)
    assert o.error() == 0
    assert_match(q_g[..., :5], q_o[..., :5], strict, "sweep")
    np.testing.assert_allclose(q_g[..., 5], q_o[..., 5], rtol=1e-13)


def test_dropin_device_pointers(cuda_device):
    import torch
    o, p, q = setup(dict(nx=16, ny=8, nz=8, boundtype=2))
    di = ev.DropIn(p, strict=True)
    sh = ev.shapes(p)
    w_o = np.zeros(sh["w"])
    o.primitive(w_o, q.copy())
    o.bound(w_o)
    w_d = torch.zeros(sh["w"], dtype=torch.float64, device=cuda_device)
    q_d = torch.from_numpy(q.copy()).to(cuda_device)
    di.primitive(w_d, q_d)
    di.bound(w_d)
    np.testing.assert_array_equal(w_d.cpu().numpy(), w_o)
    dt = di.hydrostep(w_d)
    assert dt == o.hydrostep(w_o)
    evo_d = torch.zeros(sh["evo"], dtype=torch.float64, device=cuda_device)
    s_d = torch.zeros(sh["s"], dtype=torch.float64, device=cuda_device)
    di.compevo(w_d, evo_d, s_d, dt)
    di.sweep(w_d, q_d, evo_d, s_d, dt)
    evo_o, s_o = np.zeros(sh["evo"]), np.zeros(sh["s"])
    o.compevo(w_o, evo_o, s_o, dt)
    q_o = q.copy()
    o.sweep(w_o, q_o, evo_o, s_o, dt)
    np.testing.assert_array_equal(q_d.cpu().numpy()[..., :5], q_o[..., :5])


def test_dropin_dualenergy_primitive_writes_q(cuda_device):
    kw = dict(nx=12, ny=10, nz=8, boundtype=2, dualenergy=1, de_thresh=0.3, g=5 / 3)
    o = Oracle(make_params(**kw))
    p = ev.default_params(**kw)
    q = random_q(o, np.random.default_rng(5), vel=(-2.0, 2.0))
    q[..., 5] *= 1.01   # S inconsistent with E, so both branches write back
    w_o, w_g = np.zeros(ev.shapes(p)["w"]), np.zeros(ev.shapes(p)["w"])
    qo, qg = q.copy(), q.copy()
    o.primitive(w_o, qo)
    ev.DropIn(p, strict=True).primitive(w_g, qg)
    np.testing.assert_allclose(w_g, w_o, rtol=1e-14)
    np.testing.assert_allclose(qg, qo, rtol=1e-14)
    assert not np.array_equal(qo, q)


def test_dropin_negative_pressure_raises(cuda_device):
    o, p, q = setup(dict(nx=16, ny=1, nz=1, boundtype=1))
    q[0, 0, 3, 4] = -1.0
    di = ev.DropIn(p)
    with pytest.raises(ev.EvoraError) as e:
        di.primitive(np.zeros(ev.shapes(p)["w"]), q)
    assert e.value.status & 1
