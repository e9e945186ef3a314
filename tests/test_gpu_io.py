"""The reference's output path on the GPU: the evora_run driver against the
oracle (dumps bit-exact in strict FP64), the post-processor on its dumps,
and snapshots gathered from the device against the host writer."""
import os

import numpy as np
import pytest

import evora_b200 as ev
from evora_b200 import io as eio
from oracle import io_oracle as orc
from oracle.oracle import Oracle, make_params

pytestmark = pytest.mark.gpu
ALL = eio.SNAP_CUT | eio.SNAP_SLICE | eio.SNAP_BOV


def random_state(p, seed=0):
    g = p.g
    rng = np.random.default_rng(seed)
    sh = (p.nz, p.ny, p.nx)
    r = rng.uniform(0.5, 2.0, sh)
    v = rng.uniform(-0.5, 0.5, sh + (3,))
    pr = rng.uniform(0.5, 2.0, sh)
    q = np.empty(sh + (6,))
    q[..., 0] = r
    q[..., 1:4] = r[..., None] * v
    q[..., 4] = 0.5 * r * (v ** 2).sum(-1) + pr / (g - 1)
    q[..., 5] = pr / r ** (g - 1)
    return q


def test_driver_shocktube_matches_oracle(cuda_device, tmp_path):
    # the reference's shock-tube test case: Sod, 1024 cells, reflecting upper
    # boundary, defaults otherwise (HLLC, minmod, CFL 0.5, g = (double)1.4f)
    para = tmp_path / "shocktube"
    para.write_text("shock tube\n$para\nnx = 1024, ny = 1, nz = 1\nxmin = 0.0, xmax = 1.0\nboundtype = 3\n"
                    "tstart= 0.0, tend= 0.2\n/\n$ic_para\ndl = 1.0, dr = 0.125, ul = 0.0, ur = -0.0, "
                    "pl = 1.0, pr = 0.1, x_diss = 0.5\ndir = 1\n/\n")
    r = eio.run(para, tmp_path, "--strict", "--entropy")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    o = Oracle(make_params(nx=1024, ny=1, nz=1, boundtype=3, tend=0.2))
    q = o.ic_shocktube(1.0, 0.0, 1.0, 0.125, -0.0, 0.1, 0.5, 1)
    assert (tmp_path / "data" / "in.000").read_bytes() == orc.dump_bytes(q)
    res = o.run(q, 10 ** 6)
    assert res["status"] == 0 and not res["go"]
    h, out = eio.read_dump(tmp_path / "data" / "out.000")
    assert h == (6, 1024, 1, 1, 1, 1)
    np.testing.assert_array_equal(out[..., :5], q[..., :5])
    np.testing.assert_allclose(out[..., 5], q[..., 5], rtol=1e-13)
    units = eio.read_units(tmp_path / "data" / "out.units")
    assert units.t == float(orc.fort_e(res["t"], 16, 8))
    # screen / log lines: one per integer of tsnap passed, 100 snapshots
    log = (tmp_path / "data" / "log").read_text().splitlines()
    assert len(log) == 101 and log[0].startswith("   0     1") and log[-1].endswith("100.0%")
    evo = (tmp_path / "data" / "evo").read_text().splitlines()
    assert evo[0].startswith("#              t              dt") and len(evo) == 1 + 101
    # totalmass = sum(q(1)) * volume, volume of the 1D box after compparameter
    # reset y and z to [0, dx] (parameter.f90:225)
    vol = ev.derived(ev.default_params(nx=1024, ny=1, nz=1)).volume
    assert vol == (1.0 / 1024) ** 2
    assert evo[1].split()[4] == orc.fort_e((1.0 * 512 + 0.125 * 512) * vol, 16, 6).strip()
    # post cs out: gas constant reread through data/parameter (1.4)
    r = eio.post("cs", "out", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    files = orc.cuts_and_slices_files(orc.Geometry(1024, 1, 1), orc.Gas(1.4), 1.0,
                                      orc.units_noncomoving(units.t, 1.4), [(1, out)], "out")
    assert sorted(os.listdir(tmp_path / "out")) == ["out.x.cut"]
    assert (tmp_path / "out" / "out.x.cut").read_bytes() == files["out.x.cut"]


def test_driver_kh_snapshots(cuda_device, tmp_path):
    para = tmp_path / "kh"
    para.write_text("&para\nsolver = 2, limiter = 2, boundtype = 2\ncfl = 0.5 , g = 1.4\n"
                    "nx = 32, ny = 32, nz = 1\nnsnap = 4\nslice = .t., cut = .t., bov = .t.\n"
                    "tstart= 0, tend= 0.1\n/\n")
    r = eio.run(para, tmp_path, "--ic", "kevinhelmholtz")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    o = Oracle(make_params(nx=32, ny=32, nz=1, g=1.4, limiter=2))
    assert (tmp_path / "data" / "in.000").read_bytes() == orc.dump_bytes(o.ic_kh2d())
    snaps = sorted(os.listdir(tmp_path / "snap"))
    names = {s.split(".")[0] for s in snaps}
    assert names == {"000", "001", "002", "003", "004"}
    # the last snapshot is taken at the last step, from the state out.000 holds
    _, q = eio.read_dump(tmp_path / "data" / "out.000")
    u = eio.read_units(tmp_path / "data" / "out.units")
    t_end = 0.1
    files = orc.snapshot_files(orc.Geometry(32, 32, 1), orc.Gas(1.4), q.copy(), orc.units_noncomoving(t_end, 1.4),
                               4, cut=True, slice_=True, bov=True)
    for name, blob in files.items():
        assert (tmp_path / "snap" / name).read_bytes() == blob, name
    assert u.t == float(orc.fort_e(t_end, 16, 8))


@pytest.mark.parametrize("precision,flags,dualenergy", [
    (ev.FP64, ev.STRICT | ev.CARRY_ENTROPY, 0),
    (ev.FP64, ev.CARRY_ENTROPY, 1),
    (ev.FP32, 0, 0),
], ids=["fp64-strict", "fp64-dual-energy", "fp32"])
def test_grid_snapshot_matches_host_writer(cuda_device, tmp_path, precision, flags, dualenergy):
    p = ev.default_params(nx=12, ny=10, nz=8, dualenergy=dualenergy, de_thresh=0.3)
    q0 = random_state(p, seed=11)
    if dualenergy:
        kin = 0.5 * (q0[..., 1:4] ** 2).sum(-1) / q0[..., 0]
        q0[..., 4] = np.where(np.arange(kin.size).reshape(kin.shape) % 4 == 0, kin * 1.3, q0[..., 4])
    u = eio.units_noncomoving(0.25, p.g)
    (tmp_path / "dev").mkdir()
    (tmp_path / "host").mkdir()
    with ev.Grid(p, precision, flags) as grid:
        grid.set_q(q0)
        q = grid.get_q()
        eio.grid_snapshot(grid, u, 3, ALL, tmp_path / "dev")
        after = grid.get_q()
    qh = eio.snapshot(p, q, u, 3, ALL, tmp_path / "host")
    dev, host = sorted(os.listdir(tmp_path / "dev")), sorted(os.listdir(tmp_path / "host"))
    assert dev == host and len(dev) == 8
    for name in dev:
        a, b = (tmp_path / "dev" / name).read_bytes(), (tmp_path / "host" / name).read_bytes()
        if dualenergy and name.endswith("temp.bovdata"):
            # the brick's dual-energy branch takes rho^(g-1) from the device
            # pow, the host writer from the C library's: one FP32 ulp at most
            fa, fb = np.frombuffer(a, np.float32), np.frombuffer(b, np.float32)
            assert np.max(np.abs(fa.view(np.int32) - fb.view(np.int32))) <= 1
        else:
            assert a == b, name
    if dualenergy:
        # the resynchronised cells are written back like the reference's
        # in-place pressure() leaves them (device pow: within an FP64 ulp)
        np.testing.assert_array_equal(after[..., :4], qh[..., :4])
        np.testing.assert_allclose(after, qh, rtol=4e-16, atol=0)
        assert not np.array_equal(after, q)
    else:
        np.testing.assert_array_equal(after, q)


@pytest.mark.parametrize("precision", [ev.FP64, ev.FP32])
def test_planes_round_trip(cuda_device, precision):
    p = ev.default_params(nx=7, ny=5, nz=4)
    q0 = random_state(p, seed=12)
    with ev.Grid(p, precision, ev.CARRY_ENTROPY) as grid:
        grid.set_q(q0)
        q = grid.get_q()
        np.testing.assert_array_equal(eio.get_plane(grid, 3, 2), q[1])
        np.testing.assert_array_equal(eio.get_plane(grid, 2, 5), q[:, 4])
        np.testing.assert_array_equal(eio.get_plane(grid, 1, 7), q[:, :, 6])
        plane = eio.get_plane(grid, 2, 3) * 1.5
        eio.set_plane(grid, 2, 3, plane)
        q2 = grid.get_q()
        expect = q.copy()
        expect[:, 2] = plane.astype(np.float32) if precision == ev.FP32 else plane
        np.testing.assert_array_equal(q2, expect)
        with pytest.raises(ev.EvoraError):
            eio.get_plane(grid, 3, 5)


def test_driver_comoving_chemistry_run(cuda_device, tmp_path):
    """The CIE build through the run driver (main.f90 with chemistry =
    .true.): initchem sets the species of the IC (in.000 carries q(12), bit
    for bit the oracle's), every step runs chem(q) with the sub-cycled
    cooling, and out.000 matches the oracle's run to the chemistry tests'
    tolerances; snapshot temperatures read the species."""
    kw = dict(nx=256, ny=1, nz=1, boundtype=3, supercomoving=1, omega0=0.3, lambda0=0.7, hubble0=70.0, box=1.0,
              zstart=10.0, zend=9.5, chemistry=1, cooling=1, g=5 / 3, cfl=0.4)
    para = tmp_path / "chem"
    para.write_text("comoving shock tube with chemistry\n$para\nnx = 256, ny = 1, nz = 1\nboundtype = 3\n"
                    "supercomoving = .true., omega0 = 0.3, lambda0 = 0.7, hubble0 = 70.0, box = 1.0\n"
                    "zstart = 10.0, zend = 9.5\nchemistry = .true., cooling = .true.\n"
                    "g = 1.6666666666666667, cfl = 0.4\nnsnap = 2, cut = .true.\n/\n"
                    "$ic_para\ndl = 1.0, dr = 0.5, ul = 0.0, ur = 0.0, pl = 1.0e-2, pr = 1.0e-3, x_diss = 0.5\n"
                    "dir = 1\n/\n")
    r = eio.run(para, tmp_path, "--strict", "--entropy")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    o = Oracle(make_params(**kw))
    q = o.ic_shocktube(1.0, 0.0, 1.0e-2, 0.5, 0.0, 1.0e-3, 0.5, 1)
    assert q.shape == (1, 1, 256, 12)
    o.initchem(q)
    assert (tmp_path / "data" / "in.000").read_bytes() == orc.dump_bytes(q)
    res = o.run(q, 10 ** 6)
    assert res["status"] == 0 and not res["go"]
    h, out = eio.read_dump(tmp_path / "data" / "out.000")
    assert h == (12, 256, 1, 1, 1, 1)
    # per field, the largest difference against the field's largest value
    # (the transverse momenta are 0; the device's exp and pow enter the
    # cooling, so the state is compared to the chemistry tests' tolerances)
    rel = lambda a, b: np.max(np.abs(a - b), axis=(0, 1, 2)) / np.maximum(np.max(np.abs(b), axis=(0, 1, 2)), 1e-300)   # noqa: E731,E501
    assert np.all(rel(out[..., :6], q[..., :6]) < 1e-9), rel(out[..., :6], q[..., :6])
    assert np.all(rel(out[..., 6:], q[..., 6:]) < 1e-8), rel(out[..., 6:], q[..., 6:])
    # snapshot 000 (tsnap = a nsnap passes no further integer before z =
    # 9.5): T = p / sum(n) temp0 of in.000's cells, within the E16.6
    # output (6 significant digits)
    assert sorted(os.listdir(tmp_path / "snap")) == ["000.x"]
    rows = np.loadtxt(tmp_path / "snap" / "000.x")
    u = eio.read_units(tmp_path / "data" / "in.units")
    cells = eio.read_dump(tmp_path / "data" / "in.000")[1][0, 0]
    kin = 0.5 * cells[:, 1] ** 2 / cells[:, 0]
    press = (5 / 3 - 1) * (cells[:, 4] - kin)
    temp = press / cells[:, 6:12].sum(-1) * u.temp0
    np.testing.assert_allclose(rows[:, 2], temp, rtol=1e-5)
    np.testing.assert_allclose(rows[:, 1], cells[:, 0], rtol=1e-5)
    # post cs on the q(12) dump: the 26-entry state vector per cell
    r = eio.post("cs", "out", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    cut = np.loadtxt(tmp_path / "out" / "out.x.cut")
    assert cut.shape == (256, 27)
    # (n number0) / (n / rho) / rho = number0 in every cell and species
    ratio = cut[:, 19:25] / cut[:, 13:19] / cut[:, 1:2]
    np.testing.assert_allclose(ratio, ratio[0, 0], rtol=1e-5)
    assert np.all(cut[:, 25] > 0.0)   # Lambda of the cooling gas


COSMO_PARA = ("$para\nnx = 32, ny = 32, nz = 32, boundtype = 2, solver = 2, limiter = 1\n"
              "g = 1.6666666666666667, cfl = 0.5\nsupercomoving = .true., gravity = .true.\n"
              "omega0 = 0.3, lambda0 = 0.7, hubble0 = 70.0, box = 20.0, fb = 0.17, c_cosmo = 0.01\n"
              "zstart = 50.0, zend = 46.0\ndualenergy = .true., de_thresh = 1.0e-3\n"
              "chemistry = .true., cooling = .true.\n/\n")
COSMO_KW = dict(nx=32, ny=32, nz=32, boundtype=2, solver=2, limiter=1, g=5 / 3, cfl=0.5, supercomoving=1, gravity=1,
                omega0=0.3, lambda0=0.7, hubble0=70.0, box=20.0, fb=0.17, c_cosmo=0.01, zstart=50.0, zend=46.0,
                dualenergy=1, de_thresh=1e-3, chemistry=1, cooling=1)


def test_driver_cosmological_box_from_a_dump(cuda_device, tmp_path):
    """The cosmological box (Zel'dovich IC, comoving gravity, dual energy,
    CIE chemistry with cooling) through evora_run with --ic dump:FILE, the
    way ic/grafic.f90 takes an external initial state: the driver's initchem
    and its whole run equal the same run through the grid API bit for bit."""
    p = ev.default_params(**COSMO_KW)
    q = ev.ic.cosmo_zeldovich(p, seed=5, slope=-2.0, sigma=0.05, temp_k=100.0)   # q(12), species by initchem
    assert q.shape == (32, 32, 32, 12)
    # the dump carries q(1:6): the driver's initchem sets the species
    eio.write_dump(tmp_path / "zeldovich.000", q[..., :6])
    para = tmp_path / "cosmo"
    para.write_text("cosmological box\n" + COSMO_PARA)
    r = eio.run(para, tmp_path, "--ic", "dump:" + str(tmp_path / "zeldovich.000"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    h, q_in = eio.read_dump(tmp_path / "data" / "in.000")
    assert h == (12, 32, 32, 32, 1, 32)
    np.testing.assert_array_equal(q_in, q)
    with ev.Grid(p, ev.FP64) as g:
        g.set_q(q)
        steps = 0
        while g.time()["go"] and steps < 100000:
            g.step(1)
            steps += 1
        assert g.status() == 0 and steps > 5
        q_grid = g.get_q()
        s, _ = g.cosmo()
    h, q_out = eio.read_dump(tmp_path / "data" / "out.000")
    assert h == (12, 32, 32, 32, 1, 32)
    np.testing.assert_array_equal(q_out, q_grid)
    assert s["redshift"] <= 46.0
    # the cold gas stays neutral; n(H) follows the density the run changed
    assert not np.array_equal(q_out[..., 6], q[..., 6])
    np.testing.assert_allclose(q_out[..., 6] / q_out[..., 0], q[..., 6] / q[..., 0], rtol=1e-12)


def test_driver_refuses_a_dump_of_another_grid(cuda_device, tmp_path):
    eio.write_dump(tmp_path / "bad.000", np.ones((4, 4, 4, 6)))
    para = tmp_path / "cosmo"
    para.write_text("cosmological box\n" + COSMO_PARA)
    r = eio.run(para, tmp_path, "--ic", "dump:" + str(tmp_path / "bad.000"))
    assert r.returncode != 0 and "do not fit" in r.stderr
