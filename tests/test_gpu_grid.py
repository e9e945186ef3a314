"""The resident grid (fused single-pass kernel, and the reference-kernel
backend) against the oracle's time loop (main.f90:109-155) on the same
inputs: bit-exact on rho, m, E in strict FP64; within 1e-12 (1 step) and
1e-10 (100 steps) relative L1 per field in default FP64; FP32 within 1e-5
relative L1 density of FP64.  Full-size checks use properties that do not
need the oracle: conservation in periodic boxes and direction symmetry."""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import random_q, rel_l1

pytestmark = pytest.mark.gpu


def run_oracle(kw, q, steps):
    o = Oracle(make_params(**kw))
    qq = q.copy()
    r = o.run(qq, steps)
    return qq, r


def run_gpu(kw, q, steps, precision=ev.FP64, flags=0):
    p = ev.default_params(**kw)
    with ev.Grid(p, precision, flags) as g:
        g.set_q(q)
        g.step(steps)
        return g.get_q(), g.time(), g.status()


STRICT_CASES = [
    dict(nx=16, ny=12, nz=10, boundtype=2),
    dict(nx=33, ny=9, nz=17, boundtype=3, limiter=2),
    dict(nx=20, ny=20, nz=12, boundtype=1, limiter=3, solver=1),
    dict(nx=40, ny=24, nz=1, boundtype=2),
    dict(nx=257, ny=1, nz=1, boundtype=3),
]


@pytest.mark.parametrize("backend", [0, ev.REFERENCE_KERNELS])
@pytest.mark.parametrize("kw", STRICT_CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_strict_fp64_bitwise(cuda_device, kw, backend):
    kw = dict(g=5 / 3, cfl=0.4, tend=10.0, **kw)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(11), rho=(0.8, 1.2), vel=(-0.2, 0.2), pres=(0.8, 1.2))
    qo, r = run_oracle(kw, q, 6)
    assert r["status"] == 0
    qg, t, st = run_gpu(kw, q, 6, flags=ev.STRICT | backend)
    assert st == 0
    assert t["k"] == r["steps"] and t["t"] == r["t"] and t["dt"] == r["dt"]
    np.testing.assert_array_equal(qg[..., :5], qo[..., :5])


def test_strict_entropy_field(cuda_device):
    kw = dict(nx=16, ny=12, nz=10, boundtype=2, g=5 / 3, cfl=0.4, tend=10.0)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(2))
    qo, r = run_oracle(kw, q, 4)
    qg, t, st = run_gpu(kw, q, 4, flags=ev.STRICT | ev.CARRY_ENTROPY)
    np.testing.assert_array_equal(qg[..., :5], qo[..., :5])
    np.testing.assert_allclose(qg[..., 5], qo[..., 5], rtol=1e-13)


def test_sod_1024_full_run(cuda_device):
    kw = dict(nx=1024, ny=1, nz=1, g=1.4, cfl=0.8, boundtype=1, tend=0.2)
    p = ev.default_params(**kw)
    q = ev.ic.shocktube(p)
    qo, r = run_oracle(kw, q, 100000)
    with ev.Grid(p, ev.FP64, ev.STRICT) as g:
        g.set_q(q)
        t = g.run()
        qg = g.get_q()
    assert r["status"] == 0 and not t["go"] and t["t"] == 0.2 == r["t"]
    assert t["k"] == r["steps"]
    np.testing.assert_array_equal(qg[..., :5], qo[..., :5])
    # default arithmetic: within 1e-12 relative L1
    with ev.Grid(p, ev.FP64) as g:
        g.set_q(q)
        g.run()
        qf = g.get_q()
    assert np.all(rel_l1(qf[..., :5], qo[..., :5]) <= 1e-12)


def test_kh3d_fp64_100_steps(cuda_device):
    kw = dict(nx=32, ny=32, nz=32, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    p = ev.default_params(**kw)
    q = ev.ic.kh3d(p)
    qo1, _ = run_oracle(kw, q, 1)
    qg1, _, st = run_gpu(kw, q, 1)
    assert st == 0
    assert np.all(rel_l1(qg1[..., :5], qo1[..., :5])[[0, 1, 2, 4]] <= 1e-12)
    qo, r = run_oracle(kw, q, 100)
    qg, t, st = run_gpu(kw, q, 100)
    assert st == 0 and t["k"] == 100
    err = rel_l1(qg[..., :5], qo[..., :5])
    assert np.all(err[[0, 1, 2, 4]] <= 1e-10), err
    # the z momentum stays zero up to round-off (vz = 0 everywhere initially)
    assert np.abs(qg[..., 3]).max() < 1e-12
    qs, ts, _ = run_gpu(kw, q, 100, flags=ev.STRICT)
    np.testing.assert_array_equal(qs[..., :5], qo[..., :5])


def test_fp32_form_error_vs_fp64(cuda_device):
    kw = dict(nx=48, ny=48, nz=48, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    p = ev.default_params(**kw)
    q = ev.ic.kh3d(p)
    q64, t64, _ = run_gpu(kw, q, 100)
    q32, t32, st = run_gpu(kw, q, 100, precision=ev.FP32)
    assert st == 0
    assert rel_l1(q32[..., :1], q64[..., :1])[0] <= 1e-5


def test_periodic_conservation_full_size(cuda_device):
    kw = dict(nx=256, ny=256, nz=256, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    p = ev.default_params(**kw)
    q = ev.ic.kh3d(p)
    for prec, tol in ((ev.FP64, 1e-13), (ev.FP32, 1e-6)):
        with ev.Grid(p, prec) as g:
            g.set_q(q)
            tot0 = g.totals()
            g.step(5)
            assert g.status() == 0
            tot = g.totals()
        scale = np.abs(q.reshape(-1, 6)).sum(0)
        assert np.all(np.abs(tot[:5] - tot0[:5]) <= tol * scale[:5]), (prec, tot - tot0)


def test_direction_symmetry_3d(cuda_device):
    outs = []
    for d in (1, 2, 3):
        n = [8, 8, 8]
        n[d - 1] = 96
        kw = dict(nx=n[0], ny=n[1], nz=n[2], g=1.4, cfl=0.4, boundtype=1, tend=0.05)
        p = ev.default_params(**kw)
        q = ev.ic.shocktube(p, direction=d)
        with ev.Grid(p, ev.FP64, ev.STRICT) as g:
            g.set_q(q)
            t = g.run()
            qg = g.get_q()
        prof = np.moveaxis(qg, (2, 1, 0)[d - 1], 0)[:, 3, 5, :5].copy()
        prof[:, [1, d]] = prof[:, [d, 1]]
        outs.append((t["k"], prof))
    assert outs[0][0] == outs[1][0] == outs[2][0]
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][1], outs[2][1])


def test_error_stops_the_grid(cuda_device):
    kw = dict(nx=64, ny=1, nz=1, boundtype=1, g=1.4, cfl=0.8, tend=1.0)
    p = ev.default_params(**kw)
    q = ev.ic.shocktube(p)
    q[0, 0, 10, 4] = -1.0
    with ev.Grid(p) as g:
        g.set_q(q)
        with pytest.raises(ev.EvoraError) as e:
            g.step(3)
        assert e.value.status & 1
        assert g.time()["k"] == 0
        np.testing.assert_array_equal(g.get_q()[..., :5], q[..., :5])


def test_autotune_keeps_state_and_time(cuda_device):
    kw = dict(nx=64, ny=48, nz=40, g=5 / 3, cfl=0.5, boundtype=2, tend=100.0)
    p = ev.default_params(**kw)
    q = ev.ic.kh3d(p)
    # 5 fields, and 6 (the entropy carried: the dual-energy kernels)
    for prec, flags in ((ev.FP64, ev.STRICT), (ev.FP64, ev.STRICT | ev.CARRY_ENTROPY), (ev.FP64, 0), (ev.FP32, 0),
                        (ev.FP64, ev.CARRY_ENTROPY), (ev.FP32, ev.CARRY_ENTROPY)):
        with ev.Grid(p, prec, flags) as g:
            g.set_q(q)
            g.step(2)
            before, t0 = g.get_q(), g.time()
            chosen, ms = g.autotune(reps=2)
            assert 0 <= chosen < len(ms) and all(m > 0 for m in ms)
            np.testing.assert_array_equal(g.get_q(), before)
            assert g.time() == t0
            g.step(3)
        # every tile shape gives the same answer: bit for bit in strict FP64
        # and with the FP32 state; in default FP64, whose kernels contract
        # products into FMAs per instantiation, within a few ulp; the FP32
        # packed-pair kernel, whose sums are associated differently, within
        # FP32 rounding of the others
        outs = {}
        for tile in range(len(ms)):
            with ev.Grid(p, prec, flags) as g:
                g.set_tile(tile)
                g.set_q(q)
                g.step(5)
                outs[tile] = g.get_q()
        plain = [t for t in outs if not (prec == ev.FP32 and t == ev.FP32_PAIR_TILE)]
        for t in plain:
            if prec == ev.FP64 and not flags & ev.STRICT:
                a, b = outs[t], outs[plain[0]]
                assert np.all(np.abs(a - b) <= 8 * np.spacing(np.abs(b))), np.max(np.abs(a - b))
            else:
                np.testing.assert_array_equal(outs[t], outs[plain[0]])
        if prec == ev.FP32 and ev.FP32_PAIR_TILE in outs:
            a, b = outs[ev.FP32_PAIR_TILE][..., :5], outs[plain[0]][..., :5]
            assert np.all(rel_l1(a, b)[[0, 1, 2, 4]] <= 1e-6), rel_l1(a, b)
