"""The reference's file formats (include/evora_io.h, evora_b200/csrc/io.cu)
against the Python restatement in oracle/io_oracle.py, byte for byte:
dump files (write.f90:47-65), unit files (units.f90:26-159), parameter
copies (parameter.f90:267-411), snapshots (snapshot.f90:196-360) and the
post-processor's cuts and slices (post.f90:85-246).  Host code only: these
run without a GPU."""
import os
import struct

import numpy as np
import pytest

import evora_b200 as ev
from evora_b200 import io as eio
from oracle import io_oracle as orc

REF_PARA = "/root/reference/para"


def random_state(nx, ny, nz, g, seed=0, pres=(0.5, 2.0)):
    rng = np.random.default_rng(seed)
    sh = (nz, ny, nx)
    r = rng.uniform(0.5, 2.0, sh)
    v = rng.uniform(-0.5, 0.5, sh + (3,))
    p = rng.uniform(*pres, sh)
    q = np.empty(sh + (6,))
    q[..., 0] = r
    q[..., 1:4] = r[..., None] * v
    q[..., 4] = 0.5 * r * (v ** 2).sum(-1) + p / (g - 1)
    q[..., 5] = p / r ** (g - 1)
    return q


# ------------------------------------------------------------------ format --
@pytest.mark.parametrize("x", [0.0, -0.0, 1.0, -1.0, 0.1, 123456.789, 1e-300, -2.5e-7, 9.9999999e-1,
                               0.99999995, 1e100, 7.0 / 3.0, 5e-324])
@pytest.mark.parametrize("w,d", [(16, 6), (16, 8), (12, 4), (10, 2), (12, 2)])
def test_edit_descriptor_e_matches_restatement(x, w, d, tmp_path):
    # the library's E edit descriptor, seen through the unit writer's
    # '(A16, E16.8)' lines, against the exact-decimal restatement
    if (w, d) != (16, 8):
        assert len(orc.fort_e(x, w, d)) == w
        return
    u = eio.units_noncomoving(x, 1.4)
    eio.write_units(tmp_path / "u", u)
    first = (tmp_path / "u").read_text().splitlines()[0]
    assert first == "t =".ljust(16) + orc.fort_e(x, 16, 8)


def test_fortran_e_examples():
    assert orc.fort_e(0.1, 16, 6) == "    0.100000E+00"
    assert orc.fort_e(-1.0, 12, 4) == " -0.1000E+01"
    assert orc.fort_e(0.0, 16, 6) == "    0.000000E+00"
    assert orc.fort_e(1e100, 16, 6) == "    0.100000+101"
    assert orc.fort_e(0.99999995, 16, 6) == "    0.100000E+01"
    assert orc.fort_f(12.25, 12, 1) == "        12.2"


# ------------------------------------------------------------------- dumps --
def test_dump_bytes_and_round_trip(tmp_path):
    q = random_state(7, 5, 3, 1.4, seed=1)
    path = tmp_path / "out.000"
    eio.write_dump(path, q)
    assert path.read_bytes() == orc.dump_bytes(q)
    assert eio.read_dump_header(path) == (6, 7, 5, 3, 1, 3)
    h, back = eio.read_dump(path)
    assert h == (6, 7, 5, 3, 1, 3)
    np.testing.assert_array_equal(back, q)
    # record markers: 24-byte header record, then the array
    raw = path.read_bytes()
    assert struct.unpack("<i", raw[:4])[0] == 24 and struct.unpack("<i", raw[28:32])[0] == 24
    assert struct.unpack("<i", raw[32:36])[0] == q.size * 8


def test_dump_slab_and_errors(tmp_path):
    q = random_state(4, 4, 8, 1.4, seed=2)
    eio.write_dump(tmp_path / "in.001", q[4:], lz=5, mz=8, nz=8)
    assert eio.read_dump_header(tmp_path / "in.001") == (6, 4, 4, 8, 5, 8)
    assert (tmp_path / "in.001").read_bytes() == orc.dump_bytes(q[4:], nz=8, lz=5)
    with pytest.raises(ev.EvoraError):
        eio.read_dump(tmp_path / "missing.000")
    bad = tmp_path / "bad.000"
    data = bytearray((tmp_path / "in.001").read_bytes())
    data[-1] ^= 0xFF                          # corrupt the closing marker
    bad.write_bytes(bytes(data))
    with pytest.raises(ev.EvoraError):
        eio.read_dump(bad)
    with pytest.raises(ev.EvoraError):
        eio.write_dump(tmp_path / "x", q, lz=2, mz=1)


# ------------------------------------------------------------------- units --
@pytest.mark.parametrize("g,fb", [(float(np.float32(1.4)), 1.0), (float(np.float32(5.0 / 3.0)), 0.17)])
def test_units_file(tmp_path, g, fb):
    u = eio.units_noncomoving(0.2, g, fb)
    ref = orc.units_noncomoving(0.2, g, fb)
    for k in orc.UNIT_NAMES:
        assert getattr(u, k) == ref[k], k
    eio.write_units(tmp_path / "out.units", u)
    assert (tmp_path / "out.units").read_text() == orc.units_text(ref)
    back = eio.read_units(tmp_path / "out.units")
    assert back.t == 0.2 and back.temp0 == 1.0 and back.press0 == 1.0
    assert back.jeans0 == float(orc.fort_e(ref["jeans0"], 16, 8))


# --------------------------------------------------------------- snapshots --
SNAP_CASES = [
    dict(nx=9, ny=1, nz=1),
    dict(nx=8, ny=6, nz=1),
    dict(nx=6, ny=5, nz=4, xmin=-0.5, xmax=0.5, ymin=0.0, ymax=2.0, zmin=0.0, zmax=1.0),
]


@pytest.mark.parametrize("dualenergy", [0, 1], ids=["E", "dual-energy"])
@pytest.mark.parametrize("case", SNAP_CASES, ids=["1d", "2d", "3d"])
def test_host_snapshot_matches_restatement(tmp_path, case, dualenergy):
    g = float(np.float32(1.4))
    p = ev.default_params(**case, dualenergy=dualenergy, de_thresh=0.3)
    q = random_state(p.nx, p.ny, p.nz, g, seed=3)
    if dualenergy:   # make some cells take the entropy branch of pressure()
        q[..., 4] = np.where(np.arange(q[..., 4].size).reshape(q.shape[:3]) % 3 == 0,
                             q[..., 4] * 0.6, q[..., 4])
        q[..., 4] = np.maximum(q[..., 4], 0.5 * (q[..., 1:4] ** 2).sum(-1) / q[..., 0] * 1.2)
    u = eio.units_noncomoving(0.125, g)
    out = eio.snapshot(p, q, u, 7, eio.SNAP_CUT | eio.SNAP_SLICE | eio.SNAP_BOV, tmp_path)
    geo = orc.Geometry(p.nx, p.ny, p.nz, p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax)
    qo = q.copy()
    files = orc.snapshot_files(geo, orc.Gas(g, dualenergy, 0.3), qo, orc.units_noncomoving(0.125, g), 7,
                               cut=True, slice_=True, bov=True)
    assert sorted(os.listdir(tmp_path)) == sorted(files)
    for name, data in files.items():
        assert (tmp_path / name).read_bytes() == data, name
    np.testing.assert_array_equal(out, qo)
    if not dualenergy:
        np.testing.assert_array_equal(out, q)


@pytest.mark.parametrize("case", SNAP_CASES, ids=["1d", "2d", "3d"])
def test_host_snapshot_with_chemistry_matches_restatement(tmp_path, case):
    """The CIE build's q(12): temperatures p / sum(q(7:12)) temp0
    (press2temp, comp.f90:87-102), cells read with the stride 12."""
    g = float(np.float32(1.4))
    p = ev.default_params(**case, chemistry=1)
    q6 = random_state(p.nx, p.ny, p.nz, g, seed=5)
    rng = np.random.default_rng(6)
    q = np.concatenate([q6, rng.uniform(0.01, 1.0, q6.shape[:3] + (6,))], axis=-1)
    u = eio.units_noncomoving(0.25, g)
    out = eio.snapshot(p, q, u, 3, eio.SNAP_CUT | eio.SNAP_SLICE | eio.SNAP_BOV, tmp_path)
    geo = orc.Geometry(p.nx, p.ny, p.nz, p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax)
    files = orc.snapshot_files(geo, orc.Gas(g), q.copy(), orc.units_noncomoving(0.25, g), 3,
                               cut=True, slice_=True, bov=True)
    assert sorted(os.listdir(tmp_path)) == sorted(files)
    for name, data in files.items():
        assert (tmp_path / name).read_bytes() == data, name
    np.testing.assert_array_equal(out, q)
    # the species change the temperatures (against p / rho temp0)
    plain = orc.snapshot_files(geo, orc.Gas(g), q6.copy(), orc.units_noncomoving(0.25, g), 3, cut=True,
                               slice_=False, bov=False)
    assert plain["003.x"] != files["003.x"]


def test_xz_slice_appends_like_the_reference(tmp_path):
    p = ev.default_params(nx=4, ny=4, nz=2)
    q = random_state(4, 4, 2, p.g, seed=4)
    u = eio.units_noncomoving(0.0, p.g)
    eio.snapshot(p, q, u, 0, eio.SNAP_SLICE, tmp_path)
    once = (tmp_path / "000.xz").read_bytes()
    eio.snapshot(p, q, u, 0, eio.SNAP_SLICE, tmp_path)
    assert (tmp_path / "000.xz").read_bytes() == once + once
    assert (tmp_path / "000.xy").read_bytes().count(b"\n") == 4 * 4 + 4


def test_snapshot_negative_pressure_is_an_error(tmp_path):
    p = ev.default_params(nx=4, ny=1, nz=1)
    q = random_state(4, 1, 1, p.g, seed=5)
    q[0, 0, 2, 4] = 0.0
    with pytest.raises(ev.EvoraError) as e:
        eio.snapshot(p, q, eio.units_noncomoving(0.0, p.g), 0, eio.SNAP_CUT, tmp_path)
    assert e.value.status & 1


# ----------------------------------------------------------- cuts & slices --
POST_CASES = [
    (dict(nx=16, ny=1, nz=1), [(0, 1)]),
    (dict(nx=6, ny=6, nz=1), [(0, 1)]),
    (dict(nx=5, ny=7, nz=1), [(0, 1)]),
    (dict(nx=4, ny=4, nz=4), [(0, 2), (2, 4)]),          # two ranks' slabs
    (dict(nx=6, ny=4, nz=5, xmin=-1.0, xmax=1.0), [(0, 5)]),
]


@pytest.mark.parametrize("dualenergy", [0, 1], ids=["E", "dual-energy"])
@pytest.mark.parametrize("case,slabs", POST_CASES, ids=["1d", "2d-square", "2d", "3d-cube-2ranks", "3d"])
def test_cuts_and_slices_match_restatement(tmp_path, case, slabs, dualenergy):
    g = float(np.float32(1.4))
    p = ev.default_params(**case, dualenergy=dualenergy, de_thresh=0.2)
    q = random_state(p.nx, p.ny, p.nz, g, seed=6)
    data = tmp_path / "data"
    out = tmp_path / "out"
    data.mkdir()
    out.mkdir()
    for j, (a, b) in enumerate(slabs):
        eio.write_dump(data / f"out.{j:03d}", q[a:b], lz=a + 1, mz=b, nz=p.nz)
    u = eio.units_noncomoving(0.2, g)
    eio.cuts_and_slices(p, 1.0, u, data, "out", out)
    geo = orc.Geometry(p.nx, p.ny, p.nz, p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax)
    files = orc.cuts_and_slices_files(geo, orc.Gas(g, dualenergy, 0.2), 1.0, orc.units_noncomoving(0.2, g),
                                      [(a + 1, q[a:b]) for a, b in slabs], "out")
    assert sorted(os.listdir(out)) == sorted(files)
    for name, blob in files.items():
        assert (out / name).read_bytes() == blob, name


@pytest.mark.parametrize("background", [0, 1], ids=["collisional", "uv-background"])
def test_cuts_and_slices_with_chemistry_match_restatement(tmp_path, background):
    """post cs on the CIE build's q(12) dumps: the 26-entry state vector
    (species per density, number densities, Lambda and Gamma after
    cieabundance at each cell's T, with a UV background through the
    electron-density root) byte for byte against the restatement."""
    import ctypes
    from evora_b200 import _native
    g = 5.0 / 3.0
    kw = dict(nx=8, ny=6, nz=4, supercomoving=1, omega0=0.3, lambda0=0.7, hubble0=70.0, box=1.0, zstart=10.0,
              chemistry=1, cooling=1, background=background, bg=3, j0=1e-21, g=g)
    p = ev.default_params(**kw)
    u = _native.EvoraUnits()
    assert _native.lib().evora_compunits(ctypes.byref(p), None, ctypes.byref(u)) == 0
    ud = {n: getattr(u, n) for n in orc.UNIT_NAMES}
    rng = np.random.default_rng(8)
    sh = (p.nz, p.ny, p.nx)
    rho = rng.uniform(0.5, 2.0, sh)
    vel = rng.uniform(-0.3, 0.3, sh + (3,))
    n = rng.uniform(0.05, 1.0, sh + (6,)) * rho[..., None]
    temp = 10.0 ** rng.uniform(3.7, 6.0, sh)
    press = temp * n.sum(-1) / ud["temp0"]
    q = np.empty(sh + (12,))
    q[..., 0] = rho
    q[..., 1:4] = rho[..., None] * vel
    q[..., 4] = 0.5 * rho * (vel ** 2).sum(-1) + press / (g - 1)
    q[..., 5] = press / rho ** (g - 1)
    q[..., 6:] = n
    data, out = tmp_path / "data", tmp_path / "out"
    data.mkdir()
    out.mkdir()
    eio.write_dump(data / "out.000", q)
    eio.cuts_and_slices(p, 1.0, u, data, "out", out)
    geo = orc.Geometry(p.nx, p.ny, p.nz, p.xmin, p.xmax, p.ymin, p.ymax, p.zmin, p.zmax)
    chem = orc.post_chem(ud, cooling=True, background=background, bg=3, j0=1e-21, rhoh=p.rhoh, rhohe=p.rhohe)
    assert background == 0 or chem["uv"] > 0.0
    files = orc.cuts_and_slices_files(geo, orc.Gas(g), 1.0, ud, [(1, q)], "out", chem=chem)
    assert sorted(os.listdir(out)) == sorted(files)
    for name, blob in files.items():
        assert (out / name).read_bytes() == blob, name
    row = (out / "out.x.cut").read_text().splitlines()[1].split()
    assert len(row) == 27 and float(row[-2]) > 0.0   # x + 26 entries; Lambda of a cooling gas


def test_cuts_and_slices_checks_dimensions(tmp_path):
    p = ev.default_params(nx=8, ny=1, nz=1)
    (tmp_path / "data").mkdir()
    eio.write_dump(tmp_path / "data" / "in.000", random_state(9, 1, 1, p.g))
    with pytest.raises(ev.EvoraError):
        eio.cuts_and_slices(p, 1.0, eio.units_noncomoving(0.0, p.g), tmp_path / "data", "in", tmp_path)


# ---------------------------------------------------------------- drivers --
def para_file(path, body, group="$para", ic=None):
    text = "a parameter file\n\n" + group + "\n" + body + "\n/\n"
    if ic:
        text += "\n" + group[0] + "ic_para\n" + ic + "\n/\n"
    path.write_text(text)
    return path


def run_print(path):
    r = eio.run(path, os.path.dirname(path), "--print-params")
    return r


@pytest.mark.parametrize("group", ["$para", "&para"])
def test_driver_reads_namelist_and_writes_parameter_copy(tmp_path, group):
    f = para_file(tmp_path / "p", "secondorder = .true., \nsolver = 1, limiter = 3, boundtype = 1\n"
                  "cfl = 0.9 , g = 1.4 , atomic = .false. ! a comment with nx = 5\n"
                  "nx = 64, ny = 1, nz = 1\nxmin = 0.0, xmax = 2.0d0\nboundtype = 3\n"
                  "nsnap = 40\nslice = .t.\ntstart= 0.0, tend= 0.2", group=group)
    r = run_print(f)
    assert r.returncode == 0, r.stderr
    text = r.stdout.split("status")[0]
    assert text == orc.parameter_text(secondorder=True, solver=1, limiter=3, boundtype=3, cfl=0.9, g=1.4,
                                      nx=64, ny=1, nz=1, xmin=0.0, xmax=2.0, nsnap=40, slice=True,
                                      tstart=0.0, tend=0.2)


def test_driver_refuses_unknown_or_unsupported(tmp_path):
    r = run_print(para_file(tmp_path / "p1", "nx = 8, bogus = 3"))
    assert r.returncode != 0 and "bogus" in r.stderr
    r = eio.run(para_file(tmp_path / "p2", "nx = 8, ny = 1, nz = 1\nchemistry = .true., noncie = .true."),
                tmp_path)
    assert r.returncode != 0 and "noncie" in r.stderr
    r = run_print(para_file(tmp_path / "p3", "nx = 8, dump_redshift = 3.0, x2.0"))
    assert r.returncode != 0 and "dump_redshift" in r.stderr
    r = eio.run(tmp_path / "missing", tmp_path)
    assert r.returncode != 0 and "not found" in r.stdout


@pytest.mark.skipif(not os.path.isdir(REF_PARA), reason="reference parameter files not present")
@pytest.mark.parametrize("name", ["shocktube", "kevinhelmholtz"])
def test_driver_reads_the_reference_parameter_files(name):
    r = eio.run(os.path.join(REF_PARA, name), "/tmp", "--print-params")
    assert r.returncode == 0, r.stderr
    vals = {line[:16].strip(" ="): line[16:].strip() for line in r.stdout.splitlines()}
    if name == "shocktube":
        assert vals["nx"] == "64" and vals["boundtype"] == "3" and vals["solver"] == "2"
        assert vals["cfl"] == "0.90000000E+00" and vals["tend"] == "0.20000000E+00"
    else:
        assert vals["nx"] == "128" and vals["ny"] == "128" and vals["limiter"] == "2"
        assert vals["nsnap"] == "400" and vals["slice"] == "T" and vals["tend"] == "0.12000000E+02"
    assert vals["status"] == "0"


def test_post_rereads_parameter_copy(tmp_path):
    # evora_post reads data/parameter and data/<snapshot>.units as the
    # reference's post does; the run part needs a GPU, so write both here
    p = ev.default_params(nx=6, ny=6, nz=1, xmin=0.0, xmax=1.5)
    (tmp_path / "data").mkdir()
    (tmp_path / "data" / "parameter").write_text(orc.parameter_text(nx=6, ny=6, nz=1, xmax=1.5))
    q = random_state(6, 6, 1, p.g, seed=7)
    eio.write_dump(tmp_path / "data" / "out.000", q)
    eio.write_units(tmp_path / "data" / "out.units", eio.units_noncomoving(0.5, p.g))
    r = eio.post("cs", "out", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    geo = orc.Geometry(6, 6, 1, 0.0, 1.5)
    # like the reference's post, the gas constant is the one reread through
    # its E16.8 text: 0.14000000E+01 -> 1.4, not the run's (double)1.4f
    files = orc.cuts_and_slices_files(geo, orc.Gas(1.4), 1.0, orc.units_noncomoving(0.5, p.g), [(1, q)], "out")
    for name, blob in files.items():
        assert (tmp_path / "out" / name).read_bytes() == blob, name
    r = eio.post("bov", "out", tmp_path)
    assert r.returncode != 0
