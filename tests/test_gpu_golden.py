"""GPU runs against the golden fixtures of tests/golden/ (outputs of the
reference's own hydro path, translated from its Fortran sources): strict FP64
bit-exact on rho, m, E with the same step count, t and dt, the entropy field
to 1e-13; default FP64 within 1e-12 relative L1 per field."""
import glob
import os

import numpy as np
import pytest

import evora_b200 as ev
from helpers import rel_l1
from test_oracle_pin import FIELDS, params_of

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("backend", [0, ev.REFERENCE_KERNELS], ids=["fused", "reference-kernels"])
@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_matches_golden(cuda_device, path, backend):
    g = np.load(path)
    p = ev.default_params(**params_of(g["params"]))
    if backend and p.conduction:
        pytest.skip("conduction runs on the resident SoA state only")
    steps = int(g["steps"])
    with ev.Grid(p, ev.FP64, ev.STRICT | ev.CARRY_ENTROPY | backend) as grid:
        grid.set_q(np.ascontiguousarray(g["q0"]))
        grid.step(steps)
        t = grid.time()
        q = grid.get_q()
    assert t["k"] == steps and t["t"] == float(g["t"]) and t["dt"] == float(g["dt"])
    np.testing.assert_array_equal(q[..., :5], g["q"][..., :5])
    np.testing.assert_allclose(q[..., 5], g["q"][..., 5], rtol=1e-13)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_gpu_default_fp64_close_to_golden(cuda_device, path):
    g = np.load(path)
    p = ev.default_params(**params_of(g["params"]))
    with ev.Grid(p, ev.FP64) as grid:
        grid.set_q(np.ascontiguousarray(g["q0"]))
        grid.step(int(g["steps"]))
        q = grid.get_q()
    err = rel_l1(q[..., :5], g["q"][..., :5])
    nonzero = np.abs(g["q"][..., :5]).reshape(-1, 5).sum(0) > 0
    assert np.all(err[nonzero] <= 1e-12), err
