"""The request loop with continuous batching: every request's result is the
same alone and in the mix (bit for bit: a request's arithmetic does not
depend on its neighbours), matches the oracle in strict FP64, and a tight
HBM budget only delays admission."""
import numpy as np
import pytest

import evora_b200 as ev
from evora_b200.serving import DONE, Server
from oracle.oracle import Oracle, make_params

pytestmark = pytest.mark.gpu


def mix(seed=1):
    rng = np.random.default_rng(seed)
    reqs = []
    lengths, tq = ev.ic.random_tubes(12, seed=seed, nmin=40, nmax=600)
    off = 0
    for n in lengths:
        reqs.append((np.ascontiguousarray(tq[off:off + n].reshape(1, 1, n, 6)), 0.02))
        off += n
    for nx in (64, 48):
        p = ev.default_params(nx=nx, ny=nx, nz=1, g=5 / 3)
        reqs.append((ev.ic.kh2d(p), 0.03))
    for n in (24, 20):
        p = ev.default_params(nx=n, ny=n, nz=n, g=5 / 3)
        reqs.append((ev.ic.kh3d(p, seed=int(rng.integers(100))), 0.03))
    order = rng.permutation(len(reqs))
    return [reqs[i] for i in order]


def base(**kw):
    return ev.default_params(g=5 / 3, cfl=0.4, boundtype=2, tstart=0.0, **kw)


def run_all(reqs, precision, flags=0, budget=150e9, spt=16, stagger=0, borrowed=False):
    """borrowed: Server.submit_borrowed, every other request with an output
    array of its own (the others read back by result())."""
    out = {}
    with Server(base(), precision, flags, hbm_budget_bytes=budget, steps_per_tick=spt, max_tube_cells=1024,
                max_tubes=64) as s:
        ids = []
        for i, (q, tend) in enumerate(reqs):
            if borrowed:
                ids.append(s.submit_borrowed(q, tend, out=np.full(q.shape, np.nan) if i % 2 == 0 else None))
            else:
                ids.append(s.submit(q, tend))
            for _ in range(stagger):
                s.tick()
        for _ in range(100000):
            a, p = s.tick()
            if a == 0 and p == 0:
                break
        for i, rid in enumerate(ids):
            r = s.result(rid)
            assert r is not None
            out[i] = r
        stats = s.stats()
    return out, stats


def test_alone_equals_mix_fp32(cuda_device):
    reqs = mix()
    together, stats = run_all(reqs, ev.FP32, stagger=1)
    assert stats["completed"] == len(reqs) and stats["p99_s"] >= stats["p50_s"] > 0
    for i in (0, 3, len(reqs) - 1, len(reqs) - 2):
        alone, _ = run_all([reqs[i]], ev.FP32)
        assert together[i][3] == 0 and alone[0][3] == 0
        assert together[i][2] == alone[0][2]
        np.testing.assert_array_equal(together[i][0][..., :5], alone[0][0][..., :5])


def test_strict_fp64_requests_match_oracle(cuda_device):
    reqs = mix(seed=2)
    res, _ = run_all(reqs, ev.FP64, flags=ev.STRICT, spt=8)
    for i, (q, tend) in enumerate(reqs):
        nz, ny, nx = q.shape[:3]
        o = Oracle(make_params(nx=nx, ny=ny, nz=nz, g=5 / 3, cfl=0.4, boundtype=2, tend=tend))
        qo = q.copy()
        r = o.run(qo, 1 << 30)
        qg, lat, steps, err = res[i]
        if r["status"]:
            assert err & r["status"]
            continue
        assert err == 0 and steps == r["steps"]
        np.testing.assert_array_equal(qg[..., :5], qo[..., :5])


def test_tight_budget_only_delays(cuda_device):
    reqs = [r for r in mix(seed=3) if r[0].shape[0] > 1 or r[0].shape[1] > 1]
    roomy, _ = run_all(reqs, ev.FP32)
    tight, _ = run_all(reqs, ev.FP32, budget=2.5e6)     # one 3D grid at a time
    for i in roomy:
        np.testing.assert_array_equal(tight[i][0], roomy[i][0])


def test_borrowed_arrays_equal_copies(cuda_device):
    """Requests whose states the server's copy threads read after submit,
    and whose results they write into the caller's arrays, give the results
    of the copying submit bit for bit; the inputs are left unchanged.  The
    512^2 request is copied in several chunks."""
    reqs = mix(seed=4)
    p = ev.default_params(nx=512, ny=512, nz=1, g=5 / 3)
    reqs.insert(3, (ev.ic.kh2d(p), 0.002))
    before = [q.copy() for q, _ in reqs]
    copied, _ = run_all(reqs, ev.FP32, stagger=1)
    lent, stats = run_all(reqs, ev.FP32, stagger=1, borrowed=True)
    assert stats["completed"] == len(reqs)
    for i in range(len(reqs)):
        np.testing.assert_array_equal(reqs[i][0], before[i])
        assert lent[i][3] == copied[i][3] == 0 and lent[i][2] == copied[i][2]
        np.testing.assert_array_equal(lent[i][0], copied[i][0])
