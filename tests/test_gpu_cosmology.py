"""Comoving coordinates on the GPU against the oracle (itself pinned bit for
bit to the reference's translated Fortran): grids whose control kernel
integrates the expansion factor with the step (cosmostep, compcosmo,
updatetime with timestepiteration, compunits; cosmology.f90, timestep.f90,
units.f90) and whose steps end with the expansion terms (cosmology.f90:53-72);
the dumps that dump_redshift raises; the drop-in expansion and the comoving
gravity source.  Time scalars and rho, m, E bit-exact in strict FP64; S
through the device pow where the reference's sweep takes one; conduction
through the device's T^2.5."""
import numpy as np
import pytest
import torch

import evora_b200 as ev
from helpers import random_q
from oracle import gravity_oracle as go
from oracle.oracle import TIME_FIELDS, Oracle, make_params

pytestmark = pytest.mark.gpu

COS = dict(supercomoving=1, omega0=1.0, lambda0=0.0, zstart=10.0, zend=9.6, dump_redshift=[9.9, 9.75])
CASES = [
    dict(nx=16, ny=14, nz=12, boundtype=2),
    dict(nx=24, ny=20, nz=1, boundtype=3, tempfloor=1, temp_fl=0.5),
    dict(nx=64, ny=1, nz=1, boundtype=1, jeansfloor=1, c_jeans=0.05),
    dict(nx=12, ny=10, nz=8, boundtype=2, conduction=1, simplekappa=1, box=1e-5),
    dict(nx=12, ny=10, nz=8, boundtype=1, dualenergy=1, de_thresh=0.3, atomic=1),
]
IDS = ["3d", "2d-tempfloor", "1d-jeansfloor", "3d-conduction", "3d-atomic-dual-energy"]


def kw_of(cfg, **extra):
    kw = dict(COS, g=5 / 3 if cfg.get("atomic") else 1.4, cfl=0.4, **cfg)
    kw.update(extra)
    return kw


def exact(cfg):
    """Configurations whose whole state is bit-exact (no pow on E's path)."""
    return not cfg.get("conduction") and not cfg.get("dualenergy")


@pytest.mark.parametrize("cfg", CASES, ids=IDS)
def test_grid_comoving_run_matches_oracle(cuda_device, cfg):
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(17), pres=(0.3, 3.0))
    q_o = q0.copy()
    ref = o.run(q_o, 400, trace=True)
    assert ref["status"] == 0 and not ref["go"]
    tr = ref["trace"]
    rtol = 0.0 if not cfg.get("conduction") else 1e-12
    with ev.Grid(ev.default_params(**kw), ev.FP64, ev.STRICT | ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        s0, d0 = g.cosmo()
        np.testing.assert_array_equal([s0["cosmo"], s0["redshift"]], [1 / 11.0, 10.0])
        for k in range(len(tr)):
            g.step(1)
            s, dump = g.cosmo()
            row = np.array([s[f] for f in TIME_FIELDS])
            np.testing.assert_allclose(row, tr[k, :7], rtol=rtol, atol=0)
            assert dump == int(tr[k, 7]), k
        t = g.time()
        q = g.get_q()
    assert not t["go"] and t["k"] == len(tr)
    if exact(cfg):
        np.testing.assert_array_equal(q[..., :5], q_o[..., :5])
        np.testing.assert_allclose(q[..., 5], q_o[..., 5], rtol=1e-13)
    else:
        np.testing.assert_allclose(q, q_o, rtol=1e-11, atol=0)


def test_dumps_hold_graph_replayed_steps(cuda_device):
    """Steps replayed from CUDA graphs stop at a raised dump until the host
    reads it; the run then goes on, and ends in the single-step state."""
    cfg = CASES[0]
    kw = kw_of(cfg)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(17), pres=(0.3, 3.0))
    q_o = q0.copy()
    tr = o.run(q_o, 400, trace=True)["trace"]
    dump_steps = [k + 1 for k in range(len(tr)) if tr[k, 7] > 0]
    assert len(dump_steps) == 2
    stream = torch.cuda.Stream()
    seen = []
    with ev.Grid(ev.default_params(**kw), ev.FP64, ev.STRICT | ev.CARRY_ENTROPY, stream=stream) as g:
        g.set_q(q0)
        g.step(32)
        assert g.time()["k"] == dump_steps[0]           # held at the first dump
        g.step(8)
        assert g.time()["k"] == dump_steps[0]           # still held
        s, dump = g.cosmo()
        assert dump == 1 and abs(s["redshift"] - 9.9) < 1e-9
        seen.append(g.get_q())
        t = g.run(on_dump=lambda grid, k: seen.append((k, grid.time()["k"])))
        q = g.get_q()
    assert not t["go"] and t["k"] == len(tr)
    assert seen[1] == (2, dump_steps[1])
    np.testing.assert_array_equal(q[..., :5], q_o[..., :5])


def test_dropin_expansion_matches_oracle(cuda_device):
    for de in (0, 1):
        kw = kw_of(dict(nx=12, ny=10, nz=8), dualenergy=de, de_thresh=0.3)
        o = Oracle(make_params(**kw))
        q = random_q(o, np.random.default_rng(5), pres=(0.3, 3.0))
        if de:
            q[..., 5] *= 1.02
        s = o.time()
        s[1], s[5] = 0.37, 0.021
        q_o, q_g = q.copy(), q.copy()
        o.expansion(q_o, s)
        drop = ev.DropIn(ev.default_params(**kw), strict=True)
        drop.settime(dict(zip(TIME_FIELDS, s)))
        drop.expansion(q_g)
        if de:
            np.testing.assert_allclose(q_g, q_o, rtol=1e-14, atol=0)
        else:
            np.testing.assert_array_equal(q_g, q_o)
        assert not np.array_equal(q_o[..., 4], q[..., 4])


@pytest.mark.parametrize("shape", [(16, 12, 10), (24, 20, 1)], ids=["3d", "2d"])
def test_dropin_gravpotential_comoving_matches_numpy(cuda_device, shape):
    nx, ny, nz = shape
    kw = kw_of(dict(nx=nx, ny=ny, nz=nz, boundtype=2), gravity=1, omega0=0.3, lambda0=0.7, fb=0.15)
    p = ev.default_params(**kw)
    d = ev.derived(p)
    o = Oracle(make_params(**{k: v for k, v in kw.items() if k != "gravity"}))
    q = random_q(o, np.random.default_rng(nx))
    drop = ev.DropIn(p)
    s = drop.cosmostart()
    s["cosmo"] = 0.125
    drop.settime(s)
    phi = np.zeros((nz, ny, nx), np.complex128)
    drop.gravpotential(q, phi)
    ref = go.gravpotential(q, d.dx, comoving=(0.125, 0.3, 0.15))
    assert np.max(np.abs(phi.real - ref)) <= 1e-12 * np.max(np.abs(ref))
    src = 0.125 * 1.5 * 0.3 * (q[..., 0] / 0.15 - 1.0)
    src = src - src.mean()        # the k = 0 mode is dropped by the Green's function
    assert np.max(np.abs(go.laplacian(phi.real, d.dx) - src)) < 1e-6 * np.max(np.abs(src))


def test_grid_comoving_gravity_step_matches_oracle(cuda_device):
    """One step with gravity: the oracle's comoving step (atomic: no
    expansion terms, which follow gravity) and the numpy potential from the
    comoving source at the step's a."""
    kw = kw_of(dict(nx=16, ny=12, nz=10, boundtype=2, atomic=1), omega0=0.3, lambda0=0.7, fb=0.8)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(7))
    q1 = q0.copy()
    tr = o.run(q1, 1, trace=True)["trace"]
    dt, cosmo = tr[0, 1], tr[0, 2]
    p = ev.default_params(**kw, gravity=1)
    d = ev.derived(p)
    phi = go.gravpotential(q1, d.dx, comoving=(cosmo, 0.3, 0.8))
    ref = go.gravintegration(q1, phi, dt, d.dx, d.dy, d.dz)
    with ev.Grid(p, ev.FP64, ev.STRICT | ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        g.step(1)
        s, _ = g.cosmo()
        q = g.get_q()
    assert (s["dt"], s["cosmo"]) == (dt, cosmo)
    np.testing.assert_array_equal(q[..., 0], q1[..., 0])
    for f in range(6):
        assert np.max(np.abs(q[..., f] - ref[..., f])) <= 1e-12 * np.max(np.abs(ref[..., f])), f
    assert np.max(np.abs(ref[..., 1:4] - q1[..., 1:4])) > 1e-6 * np.max(np.abs(q1[..., 1:4]))


@pytest.mark.parametrize("dualenergy", [0, 1], ids=["plain", "dual-energy"])
def test_grid_comoving_gravity_with_expansion_matches_oracle(cuda_device, dualenergy):
    """Gravity followed directly by the expansion terms (the grid applies them
    in the integration's pass): the oracle's hydro step (the step's dt is the
    hydro limit here, far below cosmostep's), the numpy potential from the
    comoving source, then the oracle's expansion(q) at the step's time
    scalars."""
    from helpers import oracle_step
    cfg = dict(nx=16, ny=12, nz=10, boundtype=2, dualenergy=dualenergy, de_thresh=0.3)
    kw = kw_of(cfg, omega0=0.3, lambda0=0.7, fb=0.8)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(8))
    tr = o.run(q0.copy(), 1, trace=True)["trace"]
    s1 = tr[0, :7]
    o_h = Oracle(make_params(**{k: v for k, v in kw.items() if k not in COS}, tend=1e6))
    q1, dt, _ = oracle_step(o_h, q0)
    assert dt == s1[1]
    p = ev.default_params(**kw, gravity=1)
    d = ev.derived(p)
    ref = go.gravintegration(q1, go.gravpotential(q1, d.dx, comoving=(s1[2], 0.3, 0.8)), dt, d.dx, d.dy, d.dz)
    o.expansion(ref, s1)
    with ev.Grid(p, ev.FP64, ev.STRICT | ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        g.step(1)
        s, _ = g.cosmo()
        q = g.get_q()
    np.testing.assert_array_equal([s[f] for f in TIME_FIELDS], s1)
    np.testing.assert_array_equal(q[..., 0], ref[..., 0])
    for f in range(6):
        assert np.max(np.abs(q[..., f] - ref[..., f])) <= 1e-12 * np.max(np.abs(ref[..., f])), f


def _low_mode_amplitude(delta):
    """Sum of |FFT| over the six |k| = 1 modes of a periodic box."""
    f = np.abs(np.fft.fftn(delta))
    return sum(f[i] for i in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)))


@pytest.mark.parametrize("precision", [ev.FP64, ev.FP32], ids=["fp64", "fp32"])
def test_zeldovich_box_grows_as_linear_theory(cuda_device, precision):
    """A cold comoving box from the Zel'dovich IC (ic/cosmo.f90's
    construction, growing mode) in an Einstein-de Sitter universe, run with
    comoving gravity and the expansion terms from z = 50 to z = 20: the
    largest modes of the density contrast grow as the linear growth factor
    D = a, mass is conserved, and the run stops on zend."""
    # cold gas (100 K at z = 50): the entropy system of dual energy keeps the
    # pressure positive where E - kin is below a thousandth of E
    kw = dict(nx=32, ny=32, nz=32, boundtype=2, g=5 / 3, cfl=0.5, supercomoving=1, gravity=1, omega0=1.0,
              lambda0=0.0, hubble0=70.0, box=50.0, zstart=50.0, zend=20.0, fb=0.17, c_cosmo=0.02,
              dualenergy=1, de_thresh=1e-3)
    p = ev.default_params(**kw)
    q0 = ev.ic.cosmo_zeldovich(p, seed=3, sigma=0.01)
    with ev.Grid(p, precision, ev.CARRY_ENTROPY) as g:
        g.set_q(q0)
        t = g.run()
        s, _ = g.cosmo()
        q = g.get_q()
    assert not t["go"] and abs(s["redshift"] - 20.0) < 1e-9
    tol = 1e-12 if precision == ev.FP64 else 1e-5
    assert abs(q[..., 0].sum() / q0[..., 0].sum() - 1.0) < tol
    growth = _low_mode_amplitude(q[..., 0] / 0.17 - 1.0) / _low_mode_amplitude(q0[..., 0] / 0.17 - 1.0)
    expected = (1.0 + 50.0) / (1.0 + 20.0)
    assert abs(growth / expected - 1.0) < 0.03, (growth, expected, t["k"])


def test_fp32_comoving_grid_tracks_fp64(cuda_device):
    kw = kw_of(dict(nx=32, ny=32, nz=32, boundtype=2))
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(3), pres=(0.3, 3.0))
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(ev.default_params(**kw), prec, ev.CARRY_ENTROPY) as g:
            g.set_q(q0)
            t = g.run()
            out[prec] = (g.get_q(), t, g.cosmo()[0])
    assert not out[ev.FP32][1]["go"]
    assert abs(out[ev.FP32][2]["redshift"] - 9.6) < 1e-9
    d = np.abs(out[ev.FP32][0][..., :5] - out[ev.FP64][0][..., :5]).max() / np.abs(out[ev.FP64][0][..., :5]).max()
    assert d < 1e-4


@pytest.mark.parametrize("shape", [(32, 24, 16), (48, 40, 1)], ids=["3d", "2d"])
def test_fp32_dual_energy_tracks_fp64(cuda_device, shape):
    """FP32 state with dual energy (pressure() in FP64 per cell, the E/S
    write-back rounded to FP32) against the FP64 dual-energy grid, on a
    state whose thermal energy is a small fraction of E in part of the box,
    so both systems of the switch are taken."""
    nx, ny, nz = shape
    kw = dict(nx=nx, ny=ny, nz=nz, boundtype=2, g=5 / 3, cfl=0.4, tend=1e6, dualenergy=1, de_thresh=0.05)
    o = Oracle(make_params(**kw))
    q0 = random_q(o, np.random.default_rng(4), vel=(-3.0, 3.0), pres=(0.01, 1.0))
    frac = 1.0 - 0.5 * (q0[..., 1:4] ** 2).sum(-1) / q0[..., 0] / q0[..., 4]
    assert (frac < 0.05).mean() > 0.05 and (frac > 0.05).mean() > 0.5
    out = {}
    for prec in (ev.FP64, ev.FP32):
        with ev.Grid(ev.default_params(**kw), prec) as g:
            g.set_q(q0)
            g.step(10)
            assert g.status() == 0
            out[prec] = g.get_q()
    a, b = out[ev.FP32], out[ev.FP64]
    l1 = np.abs(a[..., 0] - b[..., 0]).sum() / np.abs(b[..., 0]).sum()
    assert l1 < 1e-5
    for f in (4, 5):
        assert np.abs(a[..., f] - b[..., f]).sum() / np.abs(b[..., f]).sum() < 1e-4, f


def test_driver_comoving_run_writes_the_dumps(cuda_device, tmp_path):
    """evora_run with supercomoving: data/001.000 and 002.000 at the steps
    that land on dump_redshift (main.f90:197-202), their states and the
    final one against the oracle, the units at the dump's a, and the
    comoving screen lines (snapshot.f90:141-145)."""
    from evora_b200 import io as eio
    from oracle import io_oracle as orc

    para = tmp_path / "comoving"
    para.write_text("comoving shock tube\n$para\nnx = 256, ny = 1, nz = 1\nboundtype = 3\n"
                    "supercomoving = .true., omega0 = 1.0, lambda0 = 0.0, zstart = 10.0, zend = 9.6\n"
                    "dump_redshift = 9.9, 9.75\nnsnap = 100\n/\n$ic_para\ndl = 1.0, dr = 0.125, "
                    "pl = 1.0, pr = 0.1, x_diss = 0.5\ndir = 1\n/\n")
    r = eio.run(para, tmp_path, "--strict", "--entropy")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    kw = dict(nx=256, ny=1, nz=1, boundtype=3, supercomoving=1, omega0=1.0, lambda0=0.0, zstart=10.0,
              zend=9.6, dump_redshift=[9.9, 9.75])
    o = Oracle(make_params(**kw))
    q0 = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1)
    q_end = q0.copy()
    res = o.run(q_end, 10 ** 5, trace=True)
    tr = res["trace"]
    assert res["status"] == 0 and not res["go"]
    for k4 in (1, 2):
        step = int(np.nonzero(tr[:, 7] == k4)[0][0]) + 1
        q = q0.copy()
        o.run(q, step)
        h, got = eio.read_dump(tmp_path / "data" / f"{k4:03d}.000")
        assert h == (6, 256, 1, 1, 1, 1)
        np.testing.assert_array_equal(got[..., :5], q[..., :5])
        np.testing.assert_allclose(got[..., 5], q[..., 5], rtol=1e-13)
        u = eio.read_units(tmp_path / "data" / f"{k4:03d}.units")
        assert u.redshift == float(orc.fort_e(tr[step - 1, 6], 16, 8))
        assert u.cosmo == float(orc.fort_e(tr[step - 1, 2], 16, 8))
    h, out = eio.read_dump(tmp_path / "data" / "out.000")
    np.testing.assert_array_equal(out[..., :5], q_end[..., :5])
    u = eio.read_units(tmp_path / "data" / "out.units")
    assert abs(u.redshift - 9.6) < 1e-6
    # screen fires when tsnap = a * nsnap passes k1, once per step: a = 1/11
    # at the start gives the lines k1 = 0..9 on steps 1..10
    log = (tmp_path / "data" / "log").read_text().splitlines()
    assert len(log) == 10 and all(len(line) == 4 + 6 + 12 + 12 + 12 + 12 for line in log)
    for i, line in enumerate(log):
        assert int(line[:4]) == i and int(line[4:10]) == i + 1
        assert abs(float(line[34:46]) - tr[i, 2]) <= 0.5e-4 and abs(float(line[46:58]) - tr[i, 6]) <= 0.5e-2
