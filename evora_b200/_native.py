"""ctypes binding of libevora_b200.so (the C ABI of include/evora_gpu.h).

The library is built in-tree (evora_b200/_lib/libevora_b200.so) by
`python -m evora_b200.build`.  There is no fallback: if the library cannot be
loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libevora_b200.so")

c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
NDUMP = 100   # EVORA_NDUMP (global.f90:137)


class EvoraParams(ctypes.Structure):
    """evora_params: the hydro subset of namelist &para (parameter.f90:30-37)."""

    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("solver", c_int32), ("limiter", c_int32), ("boundtype", c_int32),
        ("secondorder", c_int32), ("dualenergy", c_int32), ("atomic", c_int32),
        ("gravity", c_int32),
        ("g", c_double), ("cfl", c_double), ("de_thresh", c_double),
        ("xmin", c_double), ("xmax", c_double), ("ymin", c_double),
        ("ymax", c_double), ("zmin", c_double), ("zmax", c_double),
        ("tstart", c_double), ("tend", c_double),
        ("conduction", c_int32), ("simplekappa", c_int32), ("c_cond", c_double),
        ("tempfloor", c_int32), ("jeansfloor", c_int32), ("temp_fl", c_double), ("c_jeans", c_double),
        ("fb", c_double),
        ("supercomoving", c_int32), ("c_cosmo", c_double), ("omega0", c_double), ("lambda0", c_double),
        ("hubble0", c_double), ("box", c_double), ("zstart", c_double), ("zend", c_double),
        ("dump_redshift", c_double * NDUMP),
        ("chemistry", c_int32), ("noncie", c_int32), ("cooling", c_int32), ("background", c_int32),
        ("bg", c_int32), ("cooldt", c_int32), ("j0", c_double), ("c_chem", c_double), ("substep", c_double),
        ("rhoh", c_double), ("rhohe", c_double), ("c_cooldt", c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EvoraTime(ctypes.Structure):
    """evora_time: the time scalars of module global (global.f90:86)."""

    _fields_ = [(n, c_double) for n in ("t", "dt", "cosmo", "oldcosmo", "cosmodot", "expand", "redshift")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EvoraDerived(ctypes.Structure):
    """evora_derived: constants of compparameter (parameter.f90:164-265)."""

    _fields_ = [(n, c_double) for n in (
        "g", "g1", "g1inv", "gg1", "cfl", "de_thresh1", "dx", "dy", "dz",
        "dxinv", "dyinv", "dzinv", "x0", "y0", "z0", "volume")] + [
        ("onedimension", c_int32), ("twodimension", c_int32)]


class EvoraError(RuntimeError):
    """A nonzero status of the C ABI (bit mask of EVORA_ERR_*)."""

    NAMES = {
        1: "negative pressure (comp.f90:74-84)",
        2: "unphysical Riemann pressure (riemann.f90:61-66,111-116)",
        4: "no HLL branch (riemann.f90:87-90)",
        8: "no HLLC branch (riemann.f90:148-150)",
        16: "time step <= 0 (timestep.f90:51-55)",
        32: "unknown slope limiter",
        64: "unknown Riemann solver",
        128: "invalid argument",
        256: "CUDA error",
        512: "device allocation failed",
        1024: "timeout",
        2048: "file i/o",
        4096: "timestepiteration does not converge (timestep.f90:220-223)",
        8192: "chemistry: abundances out of range or no electron-density root (chemistry.f90, cie.f90)",
    }

    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        parts = [v for k, v in self.NAMES.items() if self.status & k]
        msg = f"{where}: status {self.status} ({'; '.join(parts) or 'unknown'})"
        if self.status & 256:
            try:
                msg += f" [{lib().evora_last_error().decode()}]"
            except Exception:  # pragma: no cover
                pass
        super().__init__(msg)


_lock = threading.Lock()
_lib = None


def _declare(L):
    P = ctypes.POINTER(EvoraParams)
    D = ctypes.POINTER(EvoraDerived)
    T = ctypes.POINTER(EvoraTime)
    G = c_void_p
    sig = {
        "evora_version": ([], ctypes.c_char_p),
        "evora_last_error": ([], ctypes.c_char_p),
        "evora_params_default": ([P], None),
        "evora_compparameter": ([P, D], c_int32),
        "evora_array_sizes": ([P, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64),
                               ctypes.POINTER(c_int64), ctypes.POINTER(c_int64)], None),
        "evora_set_params": ([P], c_int32),
        "evora_set_strict": ([c_int32], c_int32),
        "evora_set_resident": ([c_int32], c_int32),
        "evora_sync": ([c_void_p], c_int32),
        "evora_invalidate": ([c_void_p], c_int32),
        "evora_primitive": ([c_void_p, c_void_p], c_int32),
        "evora_bound": ([c_void_p], c_int32),
        "evora_hydrostep": ([c_void_p, _dp], c_int32),
        "evora_updatetime": ([ctypes.POINTER(c_int32)] * 3 + [_dp, _dp], c_int32),
        "evora_compevo": ([c_void_p, c_void_p, c_void_p, c_double], c_int32),
        "evora_sweep": ([c_void_p, c_void_p, c_void_p, c_void_p, c_double], c_int32),
        "evora_grid_create": ([P, c_int32, c_int32, ctypes.POINTER(G)], c_int32),
        "evora_grid_destroy": ([G], c_int32),
        "evora_grid_set_stream": ([G, c_void_p], c_int32),
        "evora_grid_set_q": ([G, c_void_p], c_int32),
        "evora_grid_get_q": ([G, c_void_p], c_int32),
        "evora_grid_step": ([G, c_int32, c_int32], c_int32),
        "evora_grid_time": ([G, _dp, _dp, ctypes.POINTER(c_int32), ctypes.POINTER(c_int64)], c_int32),
        "evora_grid_status": ([G], c_int32),
        "evora_grid_totals": ([G, _dp], c_int32),
        "evora_grid_autotune": ([G, c_int32, ctypes.POINTER(c_int32), _dp, c_int32], c_int32),
        "evora_grid_set_tile": ([G, c_int32], c_int32),
        "evora_grid_set_timing": ([G, c_int32], c_int32),
        "evora_grid_timing": ([G, _dp, _dp, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64)], c_int32),
        "evora_grid_timing_split": ([G, _dp, _dp, _dp, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64)], c_int32),
        "evora_grid_cosmo": ([G, T, ctypes.POINTER(c_int32)], c_int32),
        "evora_cosmostart": ([T], c_int32),
        "evora_cosmostep": ([T], c_int32),
        "evora_compcosmo": ([T], c_int32),
        "evora_updatetime_cosmo": ([ctypes.POINTER(c_int32)] * 3 + [T], c_int32),
        "evora_settime": ([T], c_int32),
        "evora_expansion": ([c_void_p], c_int32),
        "evora_peebles": ([T, _dp], c_int32),
        "evora_initchem": ([c_void_p], c_int32),
    }
    optional = set()
    for name, (args, res) in sig.items():
        try:
            fn = getattr(L, name)
        except AttributeError:
            if name in optional:
                continue
            raise
        fn.argtypes = args
        fn.restype = res
    _declare_batch(L)
    _declare_io(L)
    return L


class EvoraUnits(ctypes.Structure):
    """evora_units: the unit scales of a unit file (units.f90:92-109)."""

    NAMES = ("t", "cosmo", "redshift", "length0", "time0", "density0", "velocity0", "temp0",
             "press0", "number0", "chem0", "photo0", "cool0", "heat0", "jeans0", "jeansfloor0",
             "kappa0", "meanfreepath0")
    _fields_ = [(n, c_double) for n in NAMES]


def _declare_io(L):
    """File-format entry points of include/evora_io.h."""
    P = ctypes.POINTER(EvoraParams)
    U = ctypes.POINTER(EvoraUnits)
    G = c_void_p
    s = ctypes.c_char_p
    i32p = ctypes.POINTER(c_int32)
    sig = {
        "evora_write_dump": ([s, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32], c_int32),
        "evora_read_dump_header": ([s, i32p], c_int32),
        "evora_read_dump": ([s, i32p, c_void_p, c_int64], c_int32),
        "evora_units_noncomoving": ([c_double, c_double, c_double, U], None),
        "evora_compunits": ([P, ctypes.POINTER(EvoraTime), U], c_int32),
        "evora_write_units": ([s, U], c_int32),
        "evora_read_units": ([s, U], c_int32),
        "evora_snapshot": ([P, c_void_p, U, c_int32, c_int32, s], c_int32),
        "evora_grid_snapshot": ([G, U, c_int32, c_int32, s], c_int32),
        "evora_grid_get_plane": ([G, c_int32, c_int32, c_void_p], c_int32),
        "evora_grid_set_plane": ([G, c_int32, c_int32, c_void_p], c_int32),
        "evora_cuts_and_slices": ([P, c_double, U, s, s, s], c_int32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res


def _declare_batch(L):
    """Batched-tube and no-allocation entry points (declared when present)."""
    G = c_void_p
    sig = {
        "evora_batch_create": ([ctypes.POINTER(EvoraParams), c_int32, ctypes.POINTER(c_int32),
                                c_int32, c_int32, ctypes.POINTER(G)], c_int32),
        "evora_batch_destroy": ([G], c_int32),
        "evora_batch_set_stream": ([G, c_void_p], c_int32),
        "evora_batch_set_q": ([G, c_int32, c_void_p], c_int32),
        "evora_batch_get_q": ([G, c_int32, c_void_p], c_int32),
        "evora_batch_run": ([G, c_int32, c_int32], c_int32),
        "evora_batch_info": ([G, c_int32, _dp, _dp, ctypes.POINTER(c_int32),
                              ctypes.POINTER(c_int64), ctypes.POINTER(c_int32)], c_int32),
        "evora_batch_steps_done": ([G, ctypes.POINTER(c_int64)], c_int32),
        "evora_batch_set_tend": ([G, c_int32, c_double], c_int32),
        "evora_batch_configure": ([G, c_int32, c_int32], c_int32),
        "evora_batch_autotune": ([G, c_int32, ctypes.POINTER(c_int32), ctypes.POINTER(c_int32)], c_int32),
        "evora_hydrostep_noalloc": ([c_void_p, _dp], c_int32),
        "evora_selftest_rcp": ([c_void_p, c_void_p, c_int64], c_int32),
        "evora_selftest_exp": ([c_void_p, c_void_p, c_int64], c_int32),
        "evora_gravpotential": ([c_void_p, c_void_p], c_int32),
        "evora_gravintegration": ([c_void_p, c_void_p, c_double], c_int32),
        "evora_thermalstep": ([c_void_p, c_void_p, _dp], c_int32),
        "evora_chem": ([c_void_p], c_int32),
        "evora_coolstep": ([c_void_p, c_void_p, _dp], c_int32),
        "evora_thermalconduction": ([c_void_p, c_void_p, c_double], c_int32),
        "evora_multigrid_create": ([c_int32, c_int32, c_void_p, ctypes.POINTER(G)], c_int32),
        "evora_multigrid_destroy": ([G], c_int32),
        "evora_multigrid_add": ([G, G], c_int32),
        "evora_multigrid_remove": ([G, G], c_int32),
        "evora_multigrid_step": ([G, c_int32, c_int32], c_int32),
        "evora_multigrid_status": ([G, ctypes.POINTER(G), ctypes.POINTER(c_int32), ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.POINTER(c_int64), c_int32, ctypes.POINTER(c_int32)], c_int32),
        "evora_server_create": ([ctypes.POINTER(EvoraParams), c_int32, c_int32, c_double, c_int32, c_int32,
                                 c_int32, ctypes.POINTER(G)], c_int32),
        "evora_server_destroy": ([G], c_int32),
        "evora_server_submit": ([G, c_int32, c_int32, c_int32, c_double, c_int32, c_void_p,
                                 ctypes.POINTER(c_int64)], c_int32),
        "evora_server_submit_borrowed": ([G, c_int32, c_int32, c_int32, c_double, c_int32, c_void_p, c_void_p,
                                          ctypes.POINTER(c_int64)], c_int32),
        "evora_server_tick": ([G, ctypes.POINTER(c_int32), ctypes.POINTER(c_int32)], c_int32),
        "evora_server_result": ([G, c_int64, c_void_p, _dp, ctypes.POINTER(c_int64), ctypes.POINTER(c_int32)],
                                c_int32),
        "evora_server_stats": ([G, _dp, _dp, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64), _dp], c_int32),
        "evora_server_completed": ([G, ctypes.POINTER(c_int64), c_int32, ctypes.POINTER(c_int32)], c_int32),
        "evora_server_profile": ([G, _dp], c_int32),
        "evora_server_device_ms": ([G, _dp, _dp], c_int32),
    }
    for name, (args, res) in sig.items():
        if hasattr(L, name):
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res


def lib():
    """The loaded library; raises if it is not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m evora_b200.build` "
                    "(there is no CPU fallback)")
            _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def check(status: int, where: str):
    if status:
        raise EvoraError(status, where)
