"""The CIE chemistry build on the GPU against the oracle (itself pinned bit
for bit to the reference's Fortran translated with -DCIE): the drop-in
initchem and chem(q), grids with q(12) whose steps run the species and the
sub-cycled cooling after the hydro update, comoving coefficients per step.
The rates go through the device's exp, pow and sqrt, so results are
compared to a relative tolerance; the time scalars of comoving runs stay
bit-exact while the cooling does not change the step."""
import numpy as np
import pytest

import evora_b200 as ev
from helpers import random_q
from oracle.oracle import TIME_FIELDS, Oracle, make_params

pytestmark = pytest.mark.gpu

BASE = dict(supercomoving=1, omega0=0.3, lambda0=0.7, hubble0=70.0, box=1.0, zstart=10.0, zend=9.5,
            chemistry=1, g=5 / 3, cfl=0.4)
CASES = [
    dict(cooling=0),
    dict(cooling=1),
    dict(cooling=1, background=1, bg=1, j0=1e-21),
    dict(cooling=1, background=1, bg=3, j0=1e-21, tempfloor=1, temp_fl=5e3),
    dict(cooling=1, dualenergy=1, de_thresh=0.01, jeansfloor=1, c_jeans=0.5),
]
IDS = ["abundances", "cooling", "cooling-uv1", "cooling-uv3-tempfloor", "cooling-dual-energy-jeans"]


def kw_of(cfg, **extra):
    return dict(BASE, **cfg, **extra)


def state(o, seed):
    q = random_q(o, np.random.default_rng(seed), pres=(1e-5, 1e-2))
    o.initchem(q)
    return q


def rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_dropin_initchem_and_chem_match_oracle(cuda_device, cfg):
    kw = kw_of(cfg, nx=10, ny=8, nz=6)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(2), pres=(1e-5, 1e-2))
    drop = ev.DropIn(ev.default_params(**kw), strict=True)
    q_o, q_g = q.copy(), q.copy()
    o.initchem(q_o)
    drop.initchem(q_g)
    np.testing.assert_array_equal(q_g, q_o)
    s = o.time()
    for z in (10.0, 4.5):
        s[2], s[6] = 1.0 / (1.0 + z), z
        s[1] = 3e-3
        o.settime(s)
        drop.settime(dict(zip(TIME_FIELDS, s)))
        a, b = q_o.copy(), q_o.copy()
        o.chem_at(a, s)
        drop.chem(b)
        assert rel(b[..., :6], a[..., :6]) < 1e-12
        # with a UV background the abundances come from an electron-density
        # root found to 1e-10 relative (cie.f90:114-179)
        assert rel(b[..., 6:], a[..., 6:]) < (1e-8 if cfg.get("background") else 1e-10)
        assert not np.array_equal(a[..., 6:], q_o[..., 6:])


# STRICT grids run chem(q) in the reference's order of operations; the
# default mode's (shared powers of T, a table-driven exponential, contracted
# products, FMA-contracted hydro) holds the same tolerances
@pytest.mark.parametrize("flags", [ev.STRICT | ev.CARRY_ENTROPY, ev.CARRY_ENTROPY], ids=["strict", "default"])
@pytest.mark.parametrize("cfg", CASES[1:4], ids=IDS[1:4])
def test_grid_comoving_chemistry_run_matches_oracle(cuda_device, cfg, flags):
    kw = kw_of(cfg, nx=12, ny=10, nz=8, boundtype=2)
    o = Oracle(make_params(**kw))
    q0 = state(o, 3)
    q_o = q0.copy()
    ref = o.run(q_o, 60, trace=True)
    assert ref["status"] == 0
    tr = ref["trace"]
    with ev.Grid(ev.default_params(**kw), ev.FP64, flags) as g:
        g.set_q(q0)
        np.testing.assert_array_equal(g.get_q(), q0)          # q(12) round trip
        for k in range(len(tr)):
            g.step(1)
            s, dump = g.cosmo()
            np.testing.assert_allclose([s[f] for f in TIME_FIELDS], tr[k, :7], rtol=1e-11, atol=0)
        q = g.get_q()
    assert q.shape == q_o.shape == (8, 10, 12, 12)
    assert rel(q[..., :6], q_o[..., :6]) < 1e-9
    assert rel(q[..., 6:], q_o[..., 6:]) < 1e-8


def test_fp32_chemistry_grid_tracks_fp64(cuda_device):
    # the cooled gas keeps a thermal energy far below E: dual energy, as the
    # reference's cosmological runs use it, keeps FP32 pressures positive
    kw = kw_of(dict(cooling=1, dualenergy=1, de_thresh=0.01), nx=24, ny=20, nz=16, boundtype=2)
    kw["zend"] = 8.0
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(4), vel=(-0.02, 0.02), pres=(1e-5, 1e-2))
    o.initchem(q0)
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(ev.default_params(**kw), prec, ev.CARRY_ENTROPY) as g:
            g.set_q(q0)
            g.step(20)
            assert g.status() == 0
            out[prec] = g.get_q()
    a, b = out[ev.FP32], out[ev.FP64]
    assert np.abs(a[..., 0] - b[..., 0]).sum() / np.abs(b[..., 0]).sum() < 1e-5
    assert np.abs(a[..., 6:] - b[..., 6:]).sum() / np.abs(b[..., 6:]).sum() < 1e-4


def test_chemistry_refusals(cuda_device):
    """Combinations the CIE build leaves undefined or this build does not
    have are refused at creation."""
    for extra in (dict(noncie=1), dict(conduction=1, simplekappa=1)):
        p = ev.default_params(**kw_of(dict(cooling=1), nx=8, ny=8, nz=8, **extra))
        with pytest.raises(ev.EvoraError):
            ev.Grid(p, ev.FP64)


@pytest.mark.parametrize("cfg", CASES[1:], ids=IDS[1:])
def test_dropin_coolstep_matches_oracle(cuda_device, cfg):
    """coolstep(q,w) (timestep.f90:106-143) through the C-ABI after initchem
    and one chem: the limit and the abundances written back into q."""
    kw = kw_of(cfg, nx=10, ny=8, nz=6, cooldt=1, c_cooldt=0.3)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(4), pres=(1e-5, 1e-2))
    drop = ev.DropIn(ev.default_params(**kw), strict=True)
    q_o, q_g = q.copy(), q.copy()
    o.initchem(q_o)
    drop.initchem(q_g)
    s = o.time()
    s[1], s[2], s[6] = 2e-3, 1.0 / 8.0, 7.0
    o.settime(s)
    drop.settime(dict(zip(TIME_FIELDS, s)))
    o.chem_at(q_o, s)
    drop.chem(q_g)
    w = np.zeros(o.shape_w)
    o.primitive(w, q_o)
    o.bound(w)
    q_g[...] = q_o                      # the same state; nH, nHe from each side's chem
    dt_o = o.coolstep(q_o, w, 0.7)
    dt_g = drop.coolstep(q_g, w, 0.7)
    tol = 1e-8 if cfg.get("background") else 1e-10
    assert 0.0 < dt_o < 0.7 and abs(dt_g - dt_o) <= tol * dt_o
    np.testing.assert_array_equal(q_g[..., :6], q_o[..., :6])
    assert rel(q_g[..., 6:], q_o[..., 6:]) < tol
    h = q_g[..., 6] + q_g[..., 7]        # the last cell's nH in every cell
    np.testing.assert_allclose(h, h.flat[-1], rtol=1e-12)


@pytest.mark.parametrize("flags", [ev.STRICT | ev.CARRY_ENTROPY, ev.CARRY_ENTROPY], ids=["strict", "default"])
@pytest.mark.parametrize("cfg", CASES[1:3], ids=IDS[1:3])
def test_grid_run_with_cooling_timestep_matches_oracle(cuda_device, cfg, flags):
    """Comoving grid runs with the cooling time-step limit (main.f90:120):
    every step's dt from coolstep, its abundances feeding the next chem."""
    kw = kw_of(cfg, nx=12, ny=10, nz=8, boundtype=2, cooldt=1, c_cooldt=0.05)
    o = Oracle(make_params(**kw))
    q0 = state(o, 3)
    q_o = q0.copy()
    ref = o.run(q_o, 40, trace=True)
    assert ref["status"] == 0 and ref["steps"] > 10
    tr = ref["trace"]
    with ev.Grid(ev.default_params(**kw), ev.FP64, flags) as g:
        g.set_q(q0)
        for k in range(len(tr)):
            g.step(1)
            s, dump = g.cosmo()
            np.testing.assert_allclose([s[f] for f in TIME_FIELDS], tr[k, :7], rtol=1e-9, atol=0)
        assert g.status() == 0
        q = g.get_q()
    assert rel(q[..., :6], q_o[..., :6]) < 1e-8
    assert rel(q[..., 6:], q_o[..., 6:]) < 1e-7


NCIE_CASES = [dict(cooling=0), dict(cooling=1), dict(cooling=1, background=1, bg=1, j0=1e-21),
              dict(cooling=0, background=1, bg=3, j0=1e-21, tempfloor=1, temp_fl=5e3)]
NCIE_IDS = ["patankar", "patankar-cooling", "patankar-cooling-uv1", "patankar-uv3-tempfloor"]


@pytest.mark.parametrize("cfg", NCIE_CASES, ids=NCIE_IDS)
def test_dropin_noncie_chem_matches_oracle(cuda_device, cfg):
    """The non-equilibrium build's chem(q) (ncie's Patankar sub-cycles,
    ncie.f90:26-149) through the C-ABI, three calls in a row, each from the
    previous one's abundances."""
    kw = kw_of(dict(cfg, noncie=1), nx=10, ny=8, nz=6)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(6), pres=(1e-5, 1e-2))
    drop = ev.DropIn(ev.default_params(**kw), strict=True)
    q_o, q_g = q.copy(), q.copy()
    o.initchem(q_o)
    drop.initchem(q_g)
    np.testing.assert_array_equal(q_g, q_o)
    s = o.time()
    s[1], s[2], s[6] = 3e-3, 1.0 / 7.0, 6.0
    o.settime(s)
    drop.settime(dict(zip(TIME_FIELDS, s)))
    for _ in range(3):
        o.chem_at(q_o, s)
        drop.chem(q_g)
        assert o.error() == 0
        assert rel(q_g[..., :6], q_o[..., :6]) < 1e-10
        assert rel(q_g[..., 6:], q_o[..., 6:]) < 1e-9
    assert not np.allclose(q_o[..., 6:8].sum(-1), q_o[..., 6], rtol=1e-3)   # hydrogen ionised


def test_noncie_refusals(cuda_device):
    """The non-equilibrium build advects 12 fields through the hydro update
    and carries 11 primitives: grids, the allocation-free CFL step and the
    cooling time step (whose CIE abundances it has no use for) refuse it; the
    drop-in hydro routines, chem and initchem accept it."""
    kw = kw_of(dict(cooling=1, noncie=1, cooldt=1, c_cooldt=0.1), nx=8, ny=8, nz=8)
    p = ev.default_params(**kw)
    with pytest.raises(ev.EvoraError):
        ev.Grid(p, ev.FP64)
    drop = ev.DropIn(p, strict=True)
    o = Oracle(make_params(**kw))
    q = random_q(o, np.random.default_rng(8), pres=(1e-5, 1e-2))
    drop.initchem(q)
    drop.chem(q)
    w = np.zeros(ev.hydro.shapes(p)["w"])
    assert w.shape[-1] == 11
    with pytest.raises(ev.EvoraError):
        drop.coolstep(q, w)
    # the allocation-free CFL step refuses it too, with its own message
    import ctypes
    import torch
    from evora_b200._native import lib
    wd = torch.zeros(w.shape, dtype=torch.float64, device=cuda_device)
    dt = ctypes.c_double(1e99)
    assert lib().evora_hydrostep_noalloc(ctypes.c_void_p(wd.data_ptr()), ctypes.byref(dt)) == 128
    assert b"non-equilibrium" in lib().evora_last_error()
