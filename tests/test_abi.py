"""The C ABI library loads and exports every entry point that
include/evora_gpu.h declares; host-side parameter logic matches the
reference (readparameter defaults, compparameter).  No GPU needed."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import evora_b200 as ev
from evora_b200 import _native
from oracle.oracle import Oracle, make_params

HEADER_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = []
    for f in sorted(os.listdir(HEADER_DIR)):
        if f.endswith(".h"):
            src = open(os.path.join(HEADER_DIR, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(evora_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert "evora_sweep" in names and "evora_grid_step" in names
    L = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts():
    assert ctypes.sizeof(ev.EvoraParams) == (10 * 4 + 11 * 8 + 2 * 4 + 8 + 2 * 4 + 3 * 8 + 8 + 7 * 8 + 100 * 8
                                             + 6 * 4 + 6 * 8)
    assert ctypes.sizeof(ev.EvoraDerived) == 16 * 8 + 2 * 4
    assert ctypes.sizeof(_native.EvoraTime) == 7 * 8


def test_struct_layouts_match_the_c_header(tmp_path):
    """sizeof and field offsets of the ctypes mirrors against the C compiler's
    view of include/evora_gpu.h."""
    checks = {"evora_params": (_native.EvoraParams, ["nz", "gravity", "g", "tend", "fb", "supercomoving",
                                                     "c_cosmo", "zend", "dump_redshift", "chemistry", "cooldt",
                                                     "j0", "c_cooldt"]),
              "evora_time": (_native.EvoraTime, ["t", "redshift"]),
              "evora_derived": (ev.EvoraDerived, ["volume", "twodimension"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER_DIR}/evora_gpu.h"', "int main(void) {"]
    for st, (_, fields) in checks.items():
        lines.append(f'  printf("%zu\\n", sizeof({st}));')
        for f in fields:
            lines.append(f'  printf("%zu\\n", offsetof({st}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = []
    for st, (cls, fields) in checks.items():
        want.append(ctypes.sizeof(cls))
        want += [getattr(cls, f).offset for f in fields]
    assert got == want


def test_defaults_follow_readparameter():
    p = ev.default_params()
    assert (p.nx, p.ny, p.nz) == (32, 32, 32)
    assert (p.solver, p.limiter, p.boundtype, p.secondorder) == (2, 1, 2, 1)
    assert p.cfl == 0.5
    assert p.g == float(np.float32(1.4))
    assert (p.tstart, p.tend) == (0.0, 1.0)


@pytest.mark.parametrize("kw", [dict(nx=64, ny=1, nz=1), dict(nx=32, ny=16, nz=1, xmax=2.0),
                                dict(nx=8, ny=12, nz=10, zmin=-1.0, atomic=1),
                                dict(nx=10, ny=10, nz=10, dualenergy=1, de_thresh=0.01)])
def test_compparameter_matches_oracle(kw):
    p = ev.default_params(**kw)
    d = ev.derived(p)
    o = Oracle(make_params(**kw))
    for k in ("g", "g1", "g1inv", "gg1", "cfl", "de_thresh1", "dx", "dy", "dz", "dxinv", "dyinv",
              "dzinv", "x0", "y0", "z0", "volume"):
        assert getattr(d, k) == getattr(o.d, k), k
    assert (d.onedimension, d.twodimension) == (o.d.onedimension, o.d.twodimension)


@pytest.mark.parametrize("kw,code", [(dict(solver=3), 64), (dict(limiter=4), 32), (dict(boundtype=0), 128),
                                     (dict(nx=1), 128), (dict(ny=1, nz=4), 128)])
def test_invalid_parameters_are_rejected(kw, code):
    p = ev.default_params(**kw)
    with pytest.raises(ev.EvoraError) as e:
        ev.derived(p)
    assert e.value.status == code


def test_ic_matches_oracle():
    p = ev.default_params(nx=24, ny=8, nz=6, g=5 / 3)
    o = Oracle(make_params(nx=24, ny=8, nz=6, g=5 / 3))
    np.testing.assert_allclose(ev.ic.kh3d(p), o.ic_kh3d(42, 0.01), rtol=1e-14, atol=1e-15)
    p1 = ev.default_params(nx=64, ny=1, nz=1, g=1.4)
    o1 = Oracle(make_params(nx=64, ny=1, nz=1, g=1.4))
    a, b = ev.ic.shocktube(p1), o1.ic_shocktube(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 0.5, 1)
    np.testing.assert_array_equal(a[..., :5], b[..., :5])
    np.testing.assert_allclose(a[..., 5], b[..., 5], rtol=1e-15)   # numpy pow vs libm pow
    p2 = ev.default_params(nx=32, ny=32, nz=1)
    o2 = Oracle(make_params(nx=32, ny=32, nz=1))
    np.testing.assert_allclose(ev.ic.kh2d(p2), o2.ic_kh2d(), rtol=1e-14, atol=1e-15)
