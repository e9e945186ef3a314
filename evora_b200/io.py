"""The reference's file formats through the C ABI of include/evora_io.h.

Dump files (write.f90:26-65), unit files (units.f90:76-159), in-run
snapshots (snapshot.f90:196-360) and the post-processor's cuts and slices
(post.f90:85-246), plus the two command-line drivers built beside the
library: `evora_run` (the run of main.f90) and `evora_post` (`post cs`).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from ._native import LIB_PATH, EvoraParams, EvoraUnits, check, lib

SNAP_CUT, SNAP_SLICE, SNAP_BOV = 1, 2, 4
RUN_EXE = os.path.join(os.path.dirname(LIB_PATH), "evora_run")
POST_EXE = os.path.join(os.path.dirname(LIB_PATH), "evora_post")


def _b(path) -> bytes:
    return os.fsencode(path)


def write_dump(path, q: np.ndarray, lz: int = 1, mz: int | None = None, nz: int | None = None):
    """writedata (write.f90:47-65): q has the C shape (slab z, ny, nx, nn),
    i.e. the reference's q(nn, nx, ny, lz:mz)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    nzs, ny, nx, nn = q.shape
    mz = lz + nzs - 1 if mz is None else mz
    nz = mz if nz is None else nz
    check(lib().evora_write_dump(_b(path), q.ctypes.data, nn, nx, ny, nz, lz, mz), "write_dump")


def read_dump_header(path) -> tuple:
    h = (ctypes.c_int32 * 6)()
    check(lib().evora_read_dump_header(_b(path), h), "read_dump_header")
    return tuple(h)


def read_dump(path):
    """opendata + read (write.f90:179-214): returns (header, q) with q of
    the C shape (mz - lz + 1, ny, nx, nn)."""
    nn, nx, ny, nz, lz, mz = read_dump_header(path)
    q = np.empty((mz - lz + 1, ny, nx, nn))
    h = (ctypes.c_int32 * 6)()
    check(lib().evora_read_dump(_b(path), h, q.ctypes.data, q.size), "read_dump")
    return tuple(h), q


def units_noncomoving(t: float, g: float, fb: float = 1.0) -> EvoraUnits:
    """compunits (units.f90:26-73) of a run without comoving coordinates."""
    u = EvoraUnits()
    lib().evora_units_noncomoving(t, g, fb, ctypes.byref(u))
    return u


def write_units(path, u: EvoraUnits):
    check(lib().evora_write_units(_b(path), ctypes.byref(u)), "write_units")


def read_units(path) -> EvoraUnits:
    u = EvoraUnits()
    check(lib().evora_read_units(_b(path), ctypes.byref(u)), "read_units")
    return u


def snapshot(params: EvoraParams, q: np.ndarray, u: EvoraUnits, k3: int, what: int, directory) -> np.ndarray:
    """snapshot (snapshot.f90:196-360) of a host q into `directory`; returns
    q after the in-place pressure() resynchronisation the reference does
    with dualenergy."""
    q = np.array(q, dtype=np.float64, order="C", copy=True)
    check(lib().evora_snapshot(ctypes.byref(params), q.ctypes.data, ctypes.byref(u), k3, what,
                               _b(directory)), "snapshot")
    return q


def grid_snapshot(grid, u: EvoraUnits, k3: int, what: int, directory):
    """The same from a Grid's device-resident state."""
    check(lib().evora_grid_snapshot(grid._h, ctypes.byref(u), k3, what, _b(directory)), "grid_snapshot")


def get_plane(grid, axis: int, index: int) -> np.ndarray:
    """One plane (axis 1/2/3 = x/y/z, 1-based index) in the reference layout:
    C shape (n_slow, n_fast, 6)."""
    p = grid.params
    dims = {1: (p.nz, p.ny), 2: (p.nz, p.nx), 3: (p.ny, p.nx)}[axis]
    out = np.empty(dims + (6,))
    check(lib().evora_grid_get_plane(grid._h, axis, index, out.ctypes.data), "grid_get_plane")
    return out


def set_plane(grid, axis: int, index: int, plane: np.ndarray):
    plane = np.ascontiguousarray(plane, dtype=np.float64)
    check(lib().evora_grid_set_plane(grid._h, axis, index, plane.ctypes.data), "grid_set_plane")


def cuts_and_slices(params: EvoraParams, fb: float, u: EvoraUnits, datadir, infile: str, outdir):
    """`post cs <infile>` (post.f90:85-246)."""
    check(lib().evora_cuts_and_slices(ctypes.byref(params), fb, ctypes.byref(u), _b(datadir),
                                      infile.encode(), _b(outdir)), "cuts_and_slices")


def _exe(path):
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m evora_b200.build`")
    return path


def run(parameterfile, workdir, *options, timeout: float = 600.0) -> subprocess.CompletedProcess:
    """Runs evora_run on a parameter file in `workdir` (data/ and snap/ are
    created there)."""
    cmd = [_exe(RUN_EXE), os.path.abspath(parameterfile), "--workdir", os.fspath(workdir), *options]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)


def post(mode: str, infile: str, workdir, timeout: float = 600.0) -> subprocess.CompletedProcess:
    """Runs evora_post (`post <mode> <snapshot>`) in `workdir`."""
    cmd = [_exe(POST_EXE), mode, infile, "--workdir", os.fspath(workdir)]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
