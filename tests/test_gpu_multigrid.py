"""Multi-grid batches (evora_multigrid_*): 2D and 3D grids of uneven sizes
advanced by one control kernel, one persistent update launch over the tiles
of all grids and one closing kernel per step.  Every member's result equals
the same grid stepped alone bit for bit (same step count and times), strict
FP64 members match the oracle bit for bit on rho, m, E, grids that reach
their end time stop while the others go on, members removed from a batch
carry on alone, and grids the batch cannot take are refused."""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import random_q, rel_l1

pytestmark = pytest.mark.gpu

MIX = [
    dict(nx=64, ny=48, nz=1, boundtype=2),
    dict(nx=100, ny=37, nz=1, boundtype=1, limiter=2),        # partial tiles
    dict(nx=24, ny=20, nz=16, boundtype=3, solver=1),
    dict(nx=40, ny=40, nz=40, boundtype=2),
    dict(nx=33, ny=9, nz=17, boundtype=1),
    dict(nx=16, ny=16, nz=70, boundtype=2, limiter=3),        # several z chunks
]


def members(prec, flags, tend=10.0, seed=0):
    out = []
    for i, cfg in enumerate(MIX):
        kw = dict(g=5 / 3, cfl=0.4, tend=tend, **cfg)
        o = Oracle(make_params(**kw))
        q = random_q(o, np.random.default_rng(seed + i), rho=(0.8, 1.2), vel=(-0.3, 0.3), pres=(0.8, 1.2))
        out.append((kw, q))
    return out


def step_in_batch(mix, prec, flags, steps, only=None):
    """The mix (or member `only` of it alone) through one batch."""
    sel = list(range(len(mix))) if only is None else [only]
    grids = [ev.Grid(ev.default_params(**mix[i][0]), prec, flags) for i in sel]
    try:
        with ev.MultiGrid(prec, flags) as mg:
            for g, i in zip(grids, sel):
                g.set_q(mix[i][1])
                mg.add(g)
            for k in steps:
                mg.step(k)
            st = mg.status()
        return [(g.get_q(), g.time()) for g in grids], st
    finally:
        for g in grids:
            g.close()


@pytest.mark.parametrize("prec, flags", [(ev.FP32, 0), (ev.FP64, 0), (ev.FP64, ev.STRICT)],
                         ids=["fp32", "fp64", "fp64-strict"])
def test_multigrid_matches_alone(cuda_device, prec, flags):
    mix = members(prec, flags)
    out, st = step_in_batch(mix, prec, flags, (5, 7))
    assert all(go and err == 0 and k == 12 for go, err, k in st), st
    # each member alone in a batch: bit for bit the same as in the mix
    for i in (0, 3, 5):
        (qa, ta), = step_in_batch(mix, prec, flags, (12,), only=i)[0]
        assert out[i][1] == ta
        np.testing.assert_array_equal(out[i][0], qa)
    # against the grid stepped on its own: bit for bit in strict FP64 (no
    # FMA contraction); otherwise the two compiled kernels may contract
    # multiply-adds differently, so within rounding
    for (kw, q), (qb, tb) in zip(mix, out):
        with ev.Grid(ev.default_params(**kw), prec, flags) as g:
            g.set_tile(0)
            g.set_q(q)
            g.step(12)
            qa, ta = g.get_q(), g.time()
        assert tb["k"] == ta["k"] == 12
        if flags & ev.STRICT:
            assert tb == ta
            np.testing.assert_array_equal(qb, qa)
        else:
            tol = 1e-6 if prec == ev.FP32 else 1e-13
            assert abs(tb["t"] - ta["t"]) <= tol * ta["t"]
            assert np.all(rel_l1(qb[..., :5], qa[..., :5])[[0, 1, 2, 4]] <= tol)


def test_multigrid_strict_matches_oracle(cuda_device):
    mix = members(ev.FP64, ev.STRICT, seed=10)
    grids = [ev.Grid(ev.default_params(**kw), ev.FP64, ev.STRICT) for kw, _ in mix]
    try:
        with ev.MultiGrid(ev.FP64, ev.STRICT) as mg:
            for g, (_, q) in zip(grids, mix):
                g.set_q(q)
                mg.add(g)
            mg.step(6)
        for g, (kw, q) in zip(grids, mix):
            o = Oracle(make_params(**kw))
            qo = q.copy()
            r = o.run(qo, 6)
            assert r["status"] == 0
            t = g.time()
            assert t["k"] == 6 and t["t"] == r["t"]
            np.testing.assert_array_equal(g.get_q()[..., :5], qo[..., :5])
    finally:
        for g in grids:
            g.close()


def test_multigrid_end_times_and_removal(cuda_device):
    # members with different end times stop on their own; a member taken out
    # after a few steps continues alone as if it had never been batched
    mix = members(ev.FP64, ev.STRICT, seed=20)
    tends = [0.01, 0.02, 0.05, 0.01, 0.03, 0.02]
    grids = [ev.Grid(ev.default_params(**dict(kw, tend=te)), ev.FP64, ev.STRICT) for (kw, _), te in zip(mix, tends)]
    ref = []
    for (kw, q), te in zip(mix, tends):
        with ev.Grid(ev.default_params(**dict(kw, tend=te)), ev.FP64, ev.STRICT) as g:
            g.set_tile(0)
            g.set_q(q)
            t = g.run()
            ref.append((g.get_q(), t))
    try:
        with ev.MultiGrid(ev.FP64, ev.STRICT) as mg:
            for g, (_, q) in zip(grids, mix):
                g.set_q(q)
                mg.add(g)
            mg.step(3)
            mg.remove(grids[2])
            grids[2].run()                     # alone from here on
            for _ in range(400):
                mg.step(8)
                if not any(go for go, _, _ in mg.status()):
                    break
            assert not any(go for go, _, _ in mg.status())
        for g, (qr, tr) in zip(grids, ref):
            t = g.time()
            assert not t["go"] and t == tr
            np.testing.assert_array_equal(g.get_q(), qr)
    finally:
        for g in grids:
            g.close()


def test_multigrid_refusals(cuda_device):
    with ev.MultiGrid(ev.FP32) as mg:
        for kw, prec in ((dict(nx=64, ny=1, nz=1), ev.FP32),                  # 1D: a tube
                         (dict(nx=16, ny=16, nz=16, gravity=1), ev.FP32),      # physics after the update
                         (dict(nx=16, ny=16, nz=16), ev.FP64)):                # another precision
            with ev.Grid(ev.default_params(g=5 / 3, **kw), prec) as g:
                with pytest.raises(ev.EvoraError):
                    mg.add(g)
        with ev.Grid(ev.default_params(nx=16, ny=16, nz=16, g=5 / 3), ev.FP32) as g:
            g.set_q(ev.ic.kh3d(ev.default_params(nx=16, ny=16, nz=16, g=5 / 3)))
            mg.add(g)
            with pytest.raises(ev.EvoraError):
                g.step(1)                      # stepped by its batch only
            mg.remove(g)
            g.step(1)
