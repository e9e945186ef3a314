"""The tile program of the fused CUDA kernel (evora_b200/csrc/fused_kernel.cuh),
compiled for the host with g++ (tests/emu, one std::thread per CUDA thread,
std::barrier for __syncthreads) and without FMA contraction, must reproduce
the oracle's step bit for bit: tiling, halos, ring cells, the z march and the
boundary index maps may not change a single bit of the reference result."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle import Oracle, make_params
from helpers import oracle_step, random_q

EMU = os.path.join(os.path.dirname(__file__), "emu")


class HP(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                "nx ny nz solver limiter boundtype secondorder dualenergy onedimension twodimension".split()] + \
               [(n, ctypes.c_double) for n in "g g1 g1inv gg1 cfl de_thresh1 dx dy dz dxinv dyinv dzinv".split()] + \
               [("conduction", ctypes.c_int), ("simplekappa", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in "c_cond kappa0 temp0".split()] + \
               [("tempfloor", ctypes.c_int), ("jeansfloor", ctypes.c_int)] + \
               [(n, ctypes.c_double) for n in "temp_fl temp0inv jeansfloor0".split()]


@pytest.fixture(scope="module", params=[0, 1], ids=["march", "pipelined"])
def emu(request):
    subprocess.run(["make", "-s", "-C", EMU], check=True)
    L = ctypes.CDLL(os.path.join(EMU, "_build", "libfused_emu.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    L.emu_fused_update.argtypes = [ctypes.POINTER(HP), ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_int]
    L.emu_fused_update_cfl.argtypes = [ctypes.POINTER(HP), ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_int, dp]
    L.emu_set_pipeline.argtypes = [ctypes.c_int]
    L.emu_set_pipeline(request.param)   # the FP64 (0) and FP32 (1) schedules of the 3D march
    return L


def hp_of(o):
    h = HP()
    for k in "nx ny nz solver limiter boundtype secondorder dualenergy".split():
        setattr(h, k, getattr(o.p, k))
    h.onedimension, h.twodimension = o.d.onedimension, o.d.twodimension
    for k in "g g1 g1inv gg1 cfl de_thresh1 dx dy dz dxinv dyinv dzinv".split():
        setattr(h, k, getattr(o.d, k))
    return h


CASES = [
    # nx, ny, nz, boundtype, nf, limiter, solver, tile, secondorder
    (16, 12, 8, 2, 5, 1, 2, 0, 1),
    (13, 11, 9, 2, 5, 1, 2, 0, 1),
    (13, 11, 9, 1, 5, 1, 2, 0, 1),
    (13, 11, 9, 3, 5, 1, 2, 0, 1),
    (40, 9, 35, 3, 5, 1, 2, 1, 1),
    (16, 16, 1, 2, 5, 1, 2, 0, 1),
    (21, 13, 1, 3, 5, 1, 2, 0, 1),
    (64, 1, 1, 1, 5, 1, 2, 0, 1),
    (37, 1, 1, 3, 5, 1, 2, 0, 1),
    (13, 11, 9, 2, 6, 1, 2, 0, 1),
    (13, 11, 9, 1, 5, 2, 2, 0, 1),
    (13, 11, 9, 1, 5, 3, 1, 0, 1),
    (13, 11, 9, 3, 5, 2, 1, 0, 1),
    (21, 13, 1, 3, 6, 3, 1, 0, 1),
    (13, 11, 9, 2, 5, 1, 2, 0, 0),
    (64, 1, 1, 1, 5, 1, 2, 0, 0),
    (2, 2, 2, 2, 5, 1, 2, 0, 1),      # smallest 3D grid: ghosts wrap twice
    (2, 3, 1, 1, 6, 2, 2, 0, 1),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-bt{c[3]}-nf{c[4]}-l{c[5]}-s{c[6]}-t{c[7]}-o{c[8]}")
def test_emulated_fused_step_is_bitwise_oracle(emu, case):
    nx, ny, nz, bt, nf, lim, sol, tile, so = case
    o = Oracle(make_params(nx=nx, ny=ny, nz=nz, boundtype=bt, limiter=lim, solver=sol, g=5 / 3, cfl=0.4,
                           secondorder=so))
    q = random_q(o, np.random.default_rng(nx * 131 + ny * 7 + nz))
    q2, dt, _ = oracle_step(o, q)
    assert o.error() == 0
    n = nx * ny * nz
    qin = np.ascontiguousarray(q.reshape(n, 6).T[:nf])
    qout = np.zeros_like(qin)
    dp = ctypes.POINTER(ctypes.c_double)
    err = emu.emu_fused_update(ctypes.byref(hp_of(o)), nf, qin.ctypes.data_as(dp), qout.ctypes.data_as(dp), dt, tile)
    assert err == 0
    np.testing.assert_array_equal(qout, q2.reshape(n, 6).T[:nf])


def cfl_dt(o, s):
    """hydrostep part 2 (timestep.f90:26-57) from per-axis maxima."""
    vx, vy, vz = o.d.dx / s[0], o.d.dy / s[1], o.d.dz / s[2]
    m = vx
    if vy < m:
        m = vy
    if vz < m:
        m = vz
    v = 1e6
    if m < v:
        v = m
    return o.d.cfl * v


@pytest.mark.parametrize("case", [c for c in CASES if c[1] > 1],
                         ids=lambda c: "x".join(map(str, c[:3])) + f"-bt{c[3]}-nf{c[4]}-t{c[7]}")
def test_emulated_update_reduces_next_cfl_maxima(emu, case):
    # the maxima the update reduces over the state it writes give the next
    # step's dt exactly as hydrostep over that state does
    nx, ny, nz, bt, nf, lim, sol, tile, so = case
    o = Oracle(make_params(nx=nx, ny=ny, nz=nz, boundtype=bt, limiter=lim, solver=sol, g=5 / 3, cfl=0.4,
                           secondorder=so))
    q = random_q(o, np.random.default_rng(nx * 131 + ny * 7 + nz))
    q2, dt, _ = oracle_step(o, q)
    _, dt_next, _ = oracle_step(o, q2)
    n = nx * ny * nz
    qin = np.ascontiguousarray(q.reshape(n, 6).T[:nf])
    qout = np.zeros_like(qin)
    smax = np.zeros(3)
    dp = ctypes.POINTER(ctypes.c_double)
    err = emu.emu_fused_update_cfl(ctypes.byref(hp_of(o)), nf, qin.ctypes.data_as(dp), qout.ctypes.data_as(dp),
                                   dt, tile, smax.ctypes.data_as(dp))
    assert err == 0
    np.testing.assert_array_equal(qout, q2.reshape(n, 6).T[:nf])
    assert cfl_dt(o, smax) == dt_next


# The tensor-staged march (fused_tma.cuh) on grids of whole tiles, with the
# z march split into chunks of zc planes (0: the tile's own), against the
# oracle bit for bit, and its next-step CFL maxima.
TMA_CASES = [
    # nx, ny, nz, boundtype, nf, limiter, solver, tile, secondorder, zc
    (16, 8, 9, 2, 5, 1, 2, 2, 1, 0),
    (32, 16, 7, 1, 5, 1, 2, 2, 1, 3),
    (16, 16, 12, 3, 5, 2, 1, 2, 1, 5),
    (16, 8, 6, 2, 6, 3, 2, 2, 1, 0),
    (16, 8, 5, 3, 6, 1, 1, 2, 0, 2),
    (8, 4, 6, 2, 5, 1, 2, 0, 1, 4),
    (8, 8, 3, 1, 5, 1, 2, 0, 1, 2),
]


@pytest.fixture(scope="module")
def emu_tma():
    subprocess.run(["make", "-s", "-C", EMU], check=True)
    L = ctypes.CDLL(os.path.join(EMU, "_build", "libfused_emu.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    L.emu_fused_update_cfl.argtypes = [ctypes.POINTER(HP), ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_int, dp]
    L.emu_set_pipeline.argtypes = [ctypes.c_int]
    L.emu_set_zc.argtypes = [ctypes.c_int]
    L.emu_set_pipeline(2)
    yield L
    L.emu_set_zc(0)
    L.emu_set_pipeline(0)


@pytest.mark.parametrize("case", TMA_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-bt{c[3]}-nf{c[4]}-t{c[7]}-zc{c[9]}")
def test_emulated_tma_march_is_bitwise_oracle(emu_tma, case):
    nx, ny, nz, bt, nf, lim, sol, tile, so, zc = case
    o = Oracle(make_params(nx=nx, ny=ny, nz=nz, boundtype=bt, limiter=lim, solver=sol, g=5 / 3, cfl=0.4,
                           secondorder=so))
    q = random_q(o, np.random.default_rng(nx * 131 + ny * 7 + nz))
    q2, dt, _ = oracle_step(o, q)
    _, dt_next, _ = oracle_step(o, q2)
    assert o.error() == 0
    n = nx * ny * nz
    qin = np.ascontiguousarray(q.reshape(n, 6).T[:nf])
    qout = np.zeros_like(qin)
    smax = np.zeros(3)
    dp = ctypes.POINTER(ctypes.c_double)
    emu_tma.emu_set_zc(zc)
    err = emu_tma.emu_fused_update_cfl(ctypes.byref(hp_of(o)), nf, qin.ctypes.data_as(dp), qout.ctypes.data_as(dp),
                                       dt, tile, smax.ctypes.data_as(dp))
    assert err == 0
    np.testing.assert_array_equal(qout, q2.reshape(n, 6).T[:nf])
    assert cfl_dt(o, smax) == dt_next


# The two-cells-per-thread march (fused_pair.cuh: packed pairs, shuffles,
# the fast-form arithmetic) emulated in FP64 on grids of whole tiles: equal
# to the oracle to rounding (its sums are associated differently), with the
# next-step CFL maxima.
PAIR_CASES = [
    # nx, ny, nz, boundtype, tile, zc
    (16, 8, 9, 2, 2, 0),
    (32, 16, 7, 1, 2, 3),
    (16, 16, 12, 3, 2, 5),
    (32, 8, 6, 2, 1, 4),
    (32, 4, 5, 3, 1, 2),
]


@pytest.mark.parametrize("case", PAIR_CASES, ids=lambda c: "x".join(map(str, c[:3])) + f"-bt{c[3]}-t{c[4]}-zc{c[5]}")
def test_emulated_pair_march_matches_oracle(emu_tma, case):
    nx, ny, nz, bt, tile, zc = case
    o = Oracle(make_params(nx=nx, ny=ny, nz=nz, boundtype=bt, limiter=1, solver=2, g=5 / 3, cfl=0.4))
    q = random_q(o, np.random.default_rng(nx * 17 + ny * 5 + nz))
    q2, dt, _ = oracle_step(o, q)
    _, dt_next, _ = oracle_step(o, q2)
    assert o.error() == 0
    n = nx * ny * nz
    qin = np.ascontiguousarray(q.reshape(n, 6).T[:5])
    qout = np.zeros_like(qin)
    smax = np.zeros(3)
    dp = ctypes.POINTER(ctypes.c_double)
    emu_tma.emu_set_pipeline(3)
    emu_tma.emu_set_zc(zc)
    try:
        err = emu_tma.emu_fused_update_cfl(ctypes.byref(hp_of(o)), 5, qin.ctypes.data_as(dp),
                                           qout.ctypes.data_as(dp), dt, tile, smax.ctypes.data_as(dp))
    finally:
        emu_tma.emu_set_pipeline(2)
    assert err == 0
    ref = q2.reshape(n, 6).T[:5]
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.abs(qout - ref).max() > 0          # the pair schedule ran (fast forms differ in the last bits)
    np.testing.assert_allclose(qout, ref, rtol=0, atol=1e-12 * scale.max())
    assert abs(cfl_dt(o, smax) - dt_next) <= 1e-13 * dt_next
