"""Batched independent 1D tubes (one persistent launch, each tube staged in
shared memory) against the oracle run tube by tube: strict FP64 bit-exact on
rho, m, E with the same step count and time per tube; every tube the same
alone and in the mix; budgeted launches replayed from CUDA graphs equal to a
single run to completion; a tube that fails stops alone."""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import rel_l1

pytestmark = pytest.mark.gpu


def oracle_tube(kw, n, q):
    o = Oracle(make_params(nx=n, ny=1, nz=1, **kw))
    qq = q.reshape(1, 1, n, 6).copy()
    r = o.run(qq, 1 << 30)
    return qq.reshape(n, 6), r


@pytest.mark.parametrize("solver", [1, 2])
def test_batch_strict_matches_oracle_per_tube(cuda_device, solver):
    kw = dict(g=5 / 3, cfl=0.8, boundtype=1, solver=solver, tend=0.02)
    lengths, q = ev.ic.random_tubes(24, seed=3 + solver, nmin=16, nmax=700)
    p = ev.default_params(nx=max(lengths), ny=1, nz=1, **kw)
    with ev.Batch(p, lengths, ev.FP64, ev.STRICT) as b:
        b.set_q(q)
        err = b.run()
        out = b.get_q()
        infos = [b.info(i) for i in range(len(lengths))]
    offs = np.concatenate([[0], np.cumsum(lengths)])
    for i, n in enumerate(lengths):
        qo, r = oracle_tube(kw, n, q[offs[i]:offs[i + 1]])
        if r["status"]:
            assert infos[i]["status"] == 2 and infos[i]["err"] & r["status"]
            continue
        assert infos[i]["status"] == 1 and infos[i]["err"] == 0
        assert infos[i]["k"] == r["steps"] and infos[i]["t"] == r["t"]
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1], :5], qo[:, :5])


def test_batch_alone_equals_mix_and_graph_budget(cuda_device):
    kw = dict(g=5 / 3, cfl=0.8, boundtype=1, solver=2, tend=0.05)
    lengths, q = ev.ic.random_tubes(40, seed=11, nmin=32, nmax=900)
    p = ev.default_params(nx=max(lengths), ny=1, nz=1, **kw)
    offs = np.concatenate([[0], np.cumsum(lengths)])
    with ev.Batch(p, lengths, ev.FP32) as b:
        b.set_q(q)
        b.run()
        mix = b.get_q()
        cu = b.cell_updates()
    with ev.Batch(p, lengths, ev.FP32) as b:
        b.configure(threads=128, ctas_per_sm=3)
        b.set_q(q)
        for _ in range(10000):                 # budgeted launches (graph replay)
            b.run(max_steps=7)
            if all(b.info(i)["status"] != 0 for i in range(len(lengths))):
                break
        budget = b.get_q()
        assert b.cell_updates() == cu
    np.testing.assert_array_equal(budget, mix)
    for i in (0, 7, 39):
        with ev.Batch(p, [lengths[i]], ev.FP32) as b:
            b.set_q(np.ascontiguousarray(q[offs[i]:offs[i + 1]]))
            b.run()
            np.testing.assert_array_equal(b.get_q(), mix[offs[i]:offs[i + 1]])


@pytest.mark.parametrize("ctas_per_sm,lengths", [
    (8, [3000, 64, 5000, 1200]),   # shared capacity 333 cells: q and w in the scratch slot
    (2, [3000, 64, 2000, 1200]),   # 1423 cells; 2000: w in shared memory, q in the slot (up to 2846)
])
def test_batch_long_tubes_from_global_memory(cuda_device, ctas_per_sm, lengths):
    kw = dict(g=1.4, cfl=0.8, boundtype=3, tend=0.01)
    p = ev.default_params(nx=max(lengths), ny=1, nz=1, **kw)
    qs = []
    for n in lengths:
        pt = ev.default_params(nx=n, ny=1, nz=1, **kw)
        qs.append(ev.ic.shocktube(pt, ul=0.3).reshape(n, 6))
    q = np.ascontiguousarray(np.concatenate(qs))
    with ev.Batch(p, lengths, ev.FP64, ev.STRICT) as b:
        b.configure(threads=256, ctas_per_sm=ctas_per_sm)   # small shared capacity: long tubes go to global
        b.set_q(q)
        assert b.run() == 0
        out = b.get_q()
    offs = np.concatenate([[0], np.cumsum(lengths)])
    for i, n in enumerate(lengths):
        qo, r = oracle_tube(kw, n, qs[i])
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1], :5], qo[:, :5])


def test_batch_error_isolated(cuda_device):
    kw = dict(g=1.4, cfl=0.8, boundtype=1, tend=0.05)
    lengths = [100, 120, 140]
    p = ev.default_params(nx=140, ny=1, nz=1, **kw)
    qs = [ev.ic.shocktube(ev.default_params(nx=n, ny=1, nz=1, **kw)).reshape(n, 6) for n in lengths]
    qs[1][10, 4] = -1.0                               # negative pressure in tube 1
    q = np.ascontiguousarray(np.concatenate(qs))
    with ev.Batch(p, lengths, ev.FP64, ev.STRICT) as b:
        b.set_q(q)
        err = b.run()
        assert err & 1
        assert b.info(1)["status"] == 2 and b.info(1)["k"] == 0
        for i in (0, 2):
            inf = b.info(i)
            assert inf["status"] == 1 and inf["err"] == 0
            qo, r = oracle_tube(kw, lengths[i], qs[i])
            assert inf["k"] == r["steps"]
            np.testing.assert_array_equal(b.get_q(i)[:, :5], qo[:, :5])


def test_batch_fp32_accuracy_and_autotune(cuda_device):
    kw = dict(g=5 / 3, cfl=0.8, boundtype=1, tend=0.05)
    lengths, q = ev.ic.random_tubes(64, seed=5, nmin=64, nmax=1024)
    p = ev.default_params(nx=max(lengths), ny=1, nz=1, **kw)
    with ev.Batch(p, lengths, ev.FP64) as b:
        b.set_q(q)
        b.run()
        q64 = b.get_q()
        ok = [b.info(i)["status"] == 1 for i in range(len(lengths))]
    with ev.Batch(p, lengths, ev.FP32) as b:
        b.set_q(q)
        th, ct = b.autotune(steps=5)
        assert th in (128, 256, 512) and ct in (1, 2, 3)
        b.run()
        q32 = b.get_q()
    offs = np.concatenate([[0], np.cumsum(lengths)])
    for i in range(len(lengths)):
        if ok[i]:
            assert rel_l1(q32[offs[i]:offs[i + 1], :1], q64[offs[i]:offs[i + 1], :1])[0] < 1e-4
