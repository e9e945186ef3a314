"""evora_hydrostep_noalloc: the CFL step for callers that may not allocate
device memory (a driver that allocates everything at start-up, code running
under a memory pool or beside a stream capture).  Through the C ABI, its dt
must equal that of evora_hydrostep, which allocates its scratch, on the same
device array, for two calls in a row on different states; oversized grids
and host arrays are refused with EVORA_ERR_ARG.

This file is collected last on purpose (its name), so that a run that stops
at the first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

import evora_b200 as ev
from evora_b200._native import lib
from oracle.oracle import Oracle, make_params
from helpers import random_q

pytestmark = pytest.mark.gpu


def _noalloc(w_ptr, dt_in=1e99):
    dt = ctypes.c_double(dt_in)
    st = lib().evora_hydrostep_noalloc(ctypes.c_void_p(w_ptr), ctypes.byref(dt))
    return st, dt.value


@pytest.mark.parametrize("cfg", [dict(nx=48, ny=40, nz=36, boundtype=2),
                                 dict(nx=300, ny=1, nz=1, boundtype=3)])
def test_noalloc_hydrostep_equals_hydrostep(cuda_device, cfg):
    import torch
    kw = dict(g=5 / 3, cfl=0.5, **cfg)
    o = Oracle(make_params(**kw))
    p = ev.default_params(**kw)
    di = ev.DropIn(p)
    sh = ev.shapes(p)
    for seed in (1, 2):                       # two calls in a row, different states
        q = random_q(o, np.random.default_rng(seed), vel=(-0.3 * seed, 0.3 * seed))
        w = torch.zeros(sh["w"], dtype=torch.float64, device=cuda_device)
        qd = torch.from_numpy(q).to(cuda_device)
        di.primitive(w, qd)
        di.bound(w)
        dt_ref = di.hydrostep(w, 1e99)        # existing entry point (allocates its scratch)
        st, dt = _noalloc(w.data_ptr())
        assert st == 0
        assert dt == dt_ref
        st, dt2 = _noalloc(w.data_ptr(), 0.25 * dt_ref)   # dt_in caps the result
        assert st == 0 and dt2 == 0.25 * dt_ref


def test_noalloc_hydrostep_refusals(cuda_device):
    import torch
    ev.DropIn(ev.default_params(nx=257, ny=256, nz=256))   # 16.8 M + 65536 cells: over the cap
    w = torch.zeros(16, dtype=torch.float64, device=cuda_device)
    st, _ = _noalloc(w.data_ptr())
    assert st == 128
    assert b"exceed the maximum" in lib().evora_last_error()
    ev.DropIn(ev.default_params(nx=16, ny=8, nz=8))
    host = np.ones(ev.shapes(ev.default_params(nx=16, ny=8, nz=8))["w"])
    st, _ = _noalloc(host.ctypes.data)
    assert st == 128
    assert b"device memory" in lib().evora_last_error()
