"""Parity on the benchmark configurations themselves, at their full sizes.

The small-grid tests elsewhere pin the arithmetic; these run the exact
workloads the benchmark times, with the launch shapes it uses (the
autotuned tile, the plan-time z-chunk, thousands of CTAs), against the CPU
oracle on the same seeded inputs:

* 3D Kelvin-Helmholtz 256^3 periodic, gamma 5/3, HLLC, minmod, CFL 0.5
  (kh3d seed 42, amplitude 0.01): default FP64 within 1e-12 relative L1 per
  field after 1 step and 1e-10 after 100 steps; strict FP64 bit-exact on
  rho, m, E after 3 steps; the FP32 form within 1e-5 relative L1 density of
  the oracle after 100 steps, with the tile the autotuner picks.
* 4096 batched 1D Riemann tubes (random_tubes seed 7, 128-4096 cells,
  gamma 5/3, CFL 0.8, to t = 0.1), HLLC and HLL in strict FP64: every tube
  bit-exact on rho, m, E with the oracle's step count and end time, and the
  tubes the oracle stops on fail on the GPU with the same error bit.

The oracle runs on all host threads (the grid) or in a spawned process pool
over tubes (one tube per task), so the whole file takes a few minutes.
Reference path: muscl.f90:171-274, riemann.f90:26-288, boundary.f90:26-113,
timestep.f90:26-57.
"""
import numpy as np
import pytest

import evora_b200 as ev
from oracle.oracle import Oracle, make_params
from helpers import rel_l1

pytestmark = pytest.mark.gpu

N = 256
KH = dict(nx=N, ny=N, nz=N, g=5.0 / 3.0, cfl=0.5, boundtype=2, solver=2, limiter=1, tend=1.0e6)
# the z momentum starts at zero; its relative L1 is a ratio of round-off
KH_FIELDS = [0, 1, 2, 4]


@pytest.fixture(scope="module")
def kh_oracle():
    """The oracle's state after 1, 3 and 100 steps of the KH benchmark (the
    runs are chained: tend is far away, so only q carries over)."""
    p = ev.default_params(**KH)
    q0 = ev.ic.kh3d(p, seed=42, amp=0.01)
    o = Oracle(make_params(**KH))
    q = q0.copy()
    out = {0: q0}
    done = 0
    for k in (1, 3, 100):
        r = o.run(q, k - done)
        assert r["status"] == 0 and r["steps"] == k - done
        done = k
        out[k] = q.copy()
    return out


def gpu_run(q0, steps, precision, flags=0, autotune=False):
    p = ev.default_params(**KH)
    with ev.Grid(p, precision, flags) as g:
        g.set_q(q0)
        tile = g.autotune(reps=2)[0] if autotune else None
        g.step(steps)
        assert g.status() == 0
        assert g.time()["k"] == steps
        return g.get_q(), tile


def test_kh256_fp64_vs_oracle(cuda_device, kh_oracle):
    q1, _ = gpu_run(kh_oracle[0], 1, ev.FP64, autotune=True)
    e1 = rel_l1(q1[..., :5], kh_oracle[1][..., :5])[KH_FIELDS]
    assert np.all(e1 <= 1e-12), e1
    q100, _ = gpu_run(kh_oracle[0], 100, ev.FP64, autotune=True)
    e100 = rel_l1(q100[..., :5], kh_oracle[100][..., :5])[KH_FIELDS]
    assert np.all(e100 <= 1e-10), e100


def test_kh256_strict_fp64_bitwise(cuda_device, kh_oracle):
    q3, _ = gpu_run(kh_oracle[0], 3, ev.FP64, flags=ev.STRICT)
    np.testing.assert_array_equal(q3[..., :5], kh_oracle[3][..., :5])


def test_kh256_fp32_vs_oracle(cuda_device, kh_oracle):
    q32, tile = gpu_run(kh_oracle[0], 100, ev.FP32, autotune=True)
    assert tile is not None
    e = rel_l1(q32[..., :1], kh_oracle[100][..., :1])[0]
    assert e <= 1e-5, (e, tile)


def _oracle_tubes(kw, lengths, q):
    from oracle.oracle import run_tubes
    return run_tubes(kw, lengths, q)


@pytest.mark.parametrize("solver", [2, 1], ids=["hllc", "hll"])
def test_tubes_4096_strict_vs_oracle(cuda_device, solver):
    kw = dict(g=5.0 / 3.0, cfl=0.8, boundtype=1, solver=solver, tend=0.1)
    lengths, q = ev.ic.random_tubes(4096, seed=7, nmin=128, nmax=4096)
    ref = _oracle_tubes(kw, lengths, q)
    p = ev.default_params(nx=max(lengths), ny=1, nz=1, **kw)
    with ev.Batch(p, lengths, ev.FP64, ev.STRICT) as b:
        b.set_q(q)
        b.run()
        out = b.get_q()
        infos = [b.info(i) for i in range(len(lengths))]
    offs = np.concatenate([[0], np.cumsum(lengths)])
    failed = 0
    for i, (qo, r) in enumerate(ref):
        if r["status"]:
            failed += 1
            assert infos[i]["status"] == 2 and infos[i]["err"] & r["status"], (i, infos[i], r)
            continue
        assert infos[i]["status"] == 1 and infos[i]["err"] == 0, (i, infos[i])
        assert infos[i]["k"] == r["steps"] and infos[i]["t"] == r["t"], (i, infos[i], r)
        np.testing.assert_array_equal(out[offs[i]:offs[i + 1], :5], qo[:, :5], err_msg=f"tube {i}")
    assert failed < len(lengths) // 100
