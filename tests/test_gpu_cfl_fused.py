"""The fused update reduces the next step's CFL maxima (hydrostep,
timestep.f90:26-57) over the state it writes, and the grid then skips the
CFL kernel.  The dt it gives must be the CFL kernel's, bit for bit: a grid
forced to run the CFL kernel every step (any change of the state, here a
plane written back unchanged, makes the grid fall back to it) must produce
the same t, dt and state."""
import numpy as np
import pytest

import evora_b200 as ev
from evora_b200 import io as eio

pytestmark = pytest.mark.gpu

CASES = [
    (ev.FP32, 0, 0, (40, 24, 20)),
    (ev.FP64, 0, 0, (40, 24, 20)),
    (ev.FP64, ev.STRICT | ev.CARRY_ENTROPY, 0, (33, 17, 9)),
    (ev.FP64, ev.CARRY_ENTROPY, 1, (24, 20, 12)),
    (ev.FP32, 0, 0, (64, 48, 1)),
]


@pytest.mark.parametrize("precision,flags,dualenergy,shape", CASES,
                         ids=["fp32-3d", "fp64-3d", "fp64-strict-3d", "fp64-dual-energy", "fp32-2d"])
def test_fused_cfl_maxima_equal_cfl_kernel(cuda_device, precision, flags, dualenergy, shape):
    nx, ny, nz = shape
    p = ev.default_params(nx=nx, ny=ny, nz=nz, g=5.0 / 3.0, cfl=0.4, boundtype=2, solver=2, limiter=1,
                          dualenergy=dualenergy, de_thresh=0.05, tend=10.0)
    q0 = ev.ic.kh3d(p) if nz > 1 else ev.ic.kh2d(p)
    steps = 12
    with ev.Grid(p, precision, flags) as a:
        a.set_q(q0)
        a.step(steps)            # one graph: CFL kernel once, then the fused maxima
        ta, qa = a.time(), a.get_q()
    with ev.Grid(p, precision, flags) as b:
        b.set_q(q0)
        for _ in range(steps):
            plane = eio.get_plane(b, 3, 1)
            eio.set_plane(b, 3, 1, plane)    # state unchanged, maxima no longer current
            b.step(1)
        tb, qb = b.time(), b.get_q()
    assert ta["k"] == tb["k"] == steps
    assert ta["dt"] == tb["dt"] and ta["t"] == tb["t"]
    np.testing.assert_array_equal(qa, qb)


def test_launch_count_drops_cfl_kernel(cuda_device):
    p = ev.default_params(nx=32, ny=32, nz=32, g=5.0 / 3.0, cfl=0.4, tend=10.0)
    with ev.Grid(p, ev.FP32) as g:
        g.set_q(ev.ic.kh3d(p))
        g.set_timing(True)
        g.step(4)
        t = g.timing()
    # step 1: begin, CFL, time, update; steps 2-4: one control kernel (the
    # previous step's end, this step's begin and time) and the update; then
    # the last step's end
    assert t["launches"] == 4 + 3 * 2 + 1
