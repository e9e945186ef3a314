"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/libevora_oracle.so (the plain-C FP64 restatement of the
evora hydro update, evora_oracle.c), building it with make if it is missing.
Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py use this
module, as the checker and the CPU baseline; the product never imports it.

Array shapes follow the reference's column-major layouts read in C order:
  q   (nz, ny, nx, 6)            q(6, nx, ny, nz)                main.f90:72
  w   (nz+4, ny+4, nx+4, 5)      w(5, -1:nx+2, -1:ny+2, -1:nz+2) main.f90:73
  evo (nz+2, ny+2, nx+2, 5)      evo(5, 0:nx+1, ...)             main.f90:74
  s   (nz+2, ny+2, nx+2, 3, 5)   s(5, 3, 0:nx+1, ...)            main.f90:75
The oracle keeps one set of module-global parameters (like `use global`), so
every call works on the grid last passed to `Oracle.__init__`/`configure`.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libevora_oracle.so")
_lock = threading.Lock()
_lib = None

c_int = ctypes.c_int
c_double = ctypes.c_double
c_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
NDUMP = 100   # EVORA_NDUMP (global.f90:137)
TIME_FIELDS = ("t", "dt", "cosmo", "oldcosmo", "cosmodot", "expand", "redshift")


class OracleParams(ctypes.Structure):
    """evora_params of include/evora_gpu.h (the &para subset)."""

    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("solver", ctypes.c_int32), ("limiter", ctypes.c_int32),
        ("boundtype", ctypes.c_int32), ("secondorder", ctypes.c_int32),
        ("dualenergy", ctypes.c_int32), ("atomic", ctypes.c_int32),
        ("gravity", ctypes.c_int32),
        ("g", c_double), ("cfl", c_double), ("de_thresh", c_double),
        ("xmin", c_double), ("xmax", c_double), ("ymin", c_double),
        ("ymax", c_double), ("zmin", c_double), ("zmax", c_double),
        ("tstart", c_double), ("tend", c_double),
        ("conduction", ctypes.c_int32), ("simplekappa", ctypes.c_int32), ("c_cond", c_double),
        ("tempfloor", ctypes.c_int32), ("jeansfloor", ctypes.c_int32), ("temp_fl", c_double), ("c_jeans", c_double),
        ("fb", c_double),
        ("supercomoving", ctypes.c_int32), ("c_cosmo", c_double), ("omega0", c_double), ("lambda0", c_double),
        ("hubble0", c_double), ("box", c_double), ("zstart", c_double), ("zend", c_double),
        ("dump_redshift", c_double * NDUMP),
        ("chemistry", ctypes.c_int32), ("noncie", ctypes.c_int32), ("cooling", ctypes.c_int32),
        ("background", ctypes.c_int32), ("bg", ctypes.c_int32), ("cooldt", ctypes.c_int32),
        ("j0", c_double), ("c_chem", c_double), ("substep", c_double), ("rhoh", c_double), ("rhohe", c_double),
        ("c_cooldt", c_double),
    ]


class OracleDerived(ctypes.Structure):
    _fields_ = [(n, c_double) for n in (
        "g", "g1", "g1inv", "gg1", "cfl", "de_thresh1", "dx", "dy", "dz",
        "dxinv", "dyinv", "dzinv", "x0", "y0", "z0", "volume")] + [
        ("onedimension", ctypes.c_int32), ("twodimension", ctypes.c_int32)]


def build():
    """Compile the oracle library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(_HERE, "evora_oracle.c")
            if (not os.path.exists(_LIB_PATH)
                    or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
                build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_compparameter.argtypes = [ctypes.POINTER(OracleParams)]
            L.orc_get_derived.argtypes = [ctypes.POINTER(OracleDerived)]
            L.orc_primitive.argtypes = [_dp, _dp]
            L.orc_bound.argtypes = [_dp]
            L.orc_hydrostep.argtypes = [_dp, c_double]
            L.orc_hydrostep.restype = c_double
            L.orc_updatetime.argtypes = [ctypes.POINTER(c_int), _dp, _dp]
            L.orc_compevo.argtypes = [_dp, _dp, _dp, c_double]
            L.orc_sweep.argtypes = [_dp, _dp, _dp, _dp, c_double]
            L.orc_riemann_single.argtypes = [_dp, _dp, _dp, c_int]
            L.orc_run.argtypes = [_dp, c_int, _dp, ctypes.POINTER(c_int), _dp,
                                  ctypes.POINTER(c_int)]
            L.orc_ic_shocktube.argtypes = [_dp] + [c_double] * 7 + [c_int]
            L.orc_ic_kh2d.argtypes = [_dp]
            L.orc_ic_kh3d.argtypes = [_dp, ctypes.c_uint64, c_double]
            L.orc_set_threads.argtypes = [c_int]
            L.orc_thermalstep.argtypes = [_dp, _dp, c_double]
            L.orc_thermalstep.restype = c_double
            L.orc_thermalconduction.argtypes = [_dp, _dp, c_double]
            L.orc_coolstep.argtypes = [_dp, _dp, c_double]
            L.orc_coolstep.restype = c_double
            L.orc_chem.argtypes = [_dp]
            L.orc_run_trace.argtypes = [_dp, c_int, _dp, _dp, ctypes.POINTER(c_int), _dp,
                                        ctypes.POINTER(c_int)]
            L.orc_get_time.argtypes = [_dp]
            L.orc_cosmostep.argtypes = [_dp]
            L.orc_compcosmo.argtypes = [_dp]
            L.orc_updatetime_cosmo.argtypes = [ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_int, _dp]
            L.orc_settime.argtypes = [_dp]
            L.orc_get_units.argtypes = [_dp]
            L.orc_expansion.argtypes = [_dp, _dp]
            L.orc_peebles.argtypes = [_dp]
            L.orc_peebles.restype = c_double
            L.orc_chem_at.argtypes = [_dp, _dp]
            L.orc_initchem.argtypes = [_dp]
            L.orc_get_coef.argtypes = [_dp]
            _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def make_params(**kw) -> OracleParams:
    """Parameters with the readparameter defaults (parameter.f90:41-82),
    overridden by keyword arguments."""
    p = OracleParams()
    p.nx = p.ny = p.nz = 32
    p.solver, p.limiter, p.boundtype = 2, 1, 2
    p.secondorder, p.dualenergy, p.atomic = 1, 0, 0
    p.g = float(np.float32(1.4))
    p.cfl = 0.5
    p.de_thresh = 0.0
    p.xmin = p.ymin = p.zmin = 0.0
    p.xmax = p.ymax = p.zmax = 1.0
    p.tstart, p.tend = 0.0, 1.0
    p.conduction, p.simplekappa, p.c_cond = 0, 0, float(np.float32(0.1))
    p.tempfloor, p.jeansfloor, p.temp_fl, p.c_jeans, p.fb = 0, 0, 0.0, 0.0, 1.0
    p.supercomoving, p.c_cosmo = 0, float(np.float32(0.1))
    p.omega0, p.lambda0, p.hubble0, p.box, p.zstart, p.zend = 1.0, 0.0, 50.0, 1.0, 99.0, 0.0
    for i in range(NDUMP):
        p.dump_redshift[i] = -1.0
    p.chemistry = p.noncie = p.cooling = p.background = p.bg = p.cooldt = 0
    p.j0, p.c_chem, p.substep = 1e-21, float(np.float32(0.1)), float(np.float32(0.1))
    p.rhoh, p.rhohe, p.c_cooldt = float(np.float32(0.76)), float(np.float32(0.24)), 0.0
    for k, v in kw.items():
        if k == "dump_redshift":
            for i, z in enumerate(v):
                p.dump_redshift[i] = float(z)
            continue
        setattr(p, k, v)
    return p


class Oracle:
    """The module-global state of the oracle for one grid."""

    def __init__(self, params: OracleParams | None = None, **kw):
        self.L = lib()
        self.configure(params if params is not None else make_params(**kw))

    def configure(self, params: OracleParams):
        self.p = params
        rc = self.L.orc_compparameter(ctypes.byref(params))
        if rc:
            raise ValueError(f"oracle compparameter rejected parameters (status {rc})")
        self.d = OracleDerived()
        self.L.orc_get_derived(ctypes.byref(self.d))
        self.L.orc_clear_error()

    # -- shapes ------------------------------------------------------------
    @property
    def shape_q(self):
        p = self.p
        return (p.nz, p.ny, p.nx, 12 if p.chemistry else 6)

    @property
    def shape_w(self):
        p = self.p
        return (p.nz + 4, p.ny + 4, p.nx + 4, 5)

    @property
    def shape_evo(self):
        p = self.p
        return (p.nz + 2, p.ny + 2, p.nx + 2, 5)

    @property
    def shape_s(self):
        p = self.p
        return (p.nz + 2, p.ny + 2, p.nx + 2, 3, 5)

    def zeros_q(self):
        return np.zeros(self.shape_q)

    # -- error word --------------------------------------------------------
    def error(self) -> int:
        return int(self.L.orc_error())

    def clear_error(self):
        self.L.orc_clear_error()

    def set_threads(self, n: int):
        self.L.orc_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.L.orc_max_threads())

    # -- the reference routines --------------------------------------------
    def primitive(self, w, q):
        self.L.orc_primitive(_ptr(w), _ptr(q))

    def bound(self, w):
        self.L.orc_bound(_ptr(w))

    def hydrostep(self, w, dt_in=1e99) -> float:
        return float(self.L.orc_hydrostep(_ptr(w), float(dt_in)))

    def updatetime(self, t: float, dt: float):
        go = c_int(1)
        tt, dd = c_double(t), c_double(dt)
        self.L.orc_updatetime(ctypes.byref(go), ctypes.byref(tt), ctypes.byref(dd))
        return bool(go.value), tt.value, dd.value

    def compevo(self, w, evo, s, dt):
        self.L.orc_compevo(_ptr(w), _ptr(evo), _ptr(s), float(dt))

    def sweep(self, w, q, evo, s, dt):
        self.L.orc_sweep(_ptr(w), _ptr(q), _ptr(evo), _ptr(s), float(dt))

    def thermalstep(self, q, w, dt_in=1e99) -> float:
        """thermalstep(q,w), timestep.f90:72-104 (q resynchronised in place
        with dual energy, as the reference's pressure() call does)."""
        return float(self.L.orc_thermalstep(_ptr(q), _ptr(w), float(dt_in)))

    def coolstep(self, q, w, dt_in=1e99) -> float:
        """coolstep(q,w), timestep.f90:106-143: min(dt_in, c_cooldt times the
        smallest cooling time); q(7:12) is overwritten with the equilibrium
        abundances at the last chem/initchem cell's nH and nHe, as there."""
        return float(self.L.orc_coolstep(_ptr(q), _ptr(w), float(dt_in)))

    def chem(self, q):
        """chem(q), chemistry.f90:72-121, plain build: the pressure floors."""
        self.L.orc_chem(_ptr(q))

    def thermalconduction(self, q, w, dt):
        """thermalconduction(q,w), conduction.f90:26-122."""
        self.L.orc_thermalconduction(_ptr(q), _ptr(w), float(dt))

    def riemann(self, wl, wr, direction: int):
        wl = np.ascontiguousarray(wl, dtype=np.float64)
        wr = np.ascontiguousarray(wr, dtype=np.float64)
        f = np.zeros(6)
        self.L.orc_riemann_single(_ptr(wl), _ptr(wr), _ptr(f), int(direction))
        return f

    def run(self, q, max_steps: int, trace: bool = False):
        """The loop of main.f90:109-203 on q (in place): hydro, and the
        comoving time scalars, floors, conduction and expansion terms when
        enabled.  Returns dict(t, steps, dt, go, status), plus with trace an
        array (steps, 8): the time scalars after each updatetime (TIME_FIELDS)
        and the dump number the step raised."""
        t, dt = c_double(0.0), c_double(0.0)
        steps, go = c_int(0), c_int(0)
        tr = np.zeros((max(int(max_steps), 1), 8)) if trace else None
        st = self.L.orc_run_trace(_ptr(q), int(max_steps), _ptr(tr) if trace else None, ctypes.byref(t),
                                  ctypes.byref(steps), ctypes.byref(dt), ctypes.byref(go))
        out = dict(t=t.value, steps=steps.value, dt=dt.value, go=bool(go.value), status=int(st))
        if trace:
            out["trace"] = tr[:steps.value].copy()
        return out

    # -- comoving time scalars (7 values in TIME_FIELDS order) ---------------
    def time(self):
        s = np.zeros(7)
        self.L.orc_get_time(_ptr(s))
        return s

    def cosmostep(self, s):
        s = np.array(s, dtype=np.float64)
        self.L.orc_cosmostep(_ptr(s))
        return s

    def compcosmo(self, s):
        s = np.array(s, dtype=np.float64)
        self.L.orc_compcosmo(_ptr(s))
        return s

    def updatetime_cosmo(self, go: bool, s, k: int = 1):
        s = np.array(s, dtype=np.float64)
        g, d = c_int(1 if go else 0), c_int(0)
        self.L.orc_updatetime_cosmo(ctypes.byref(g), ctypes.byref(d), int(k), _ptr(s))
        return bool(g.value), bool(d.value), s

    def settime(self, s):
        """Sets the time scalars and recomputes the units (compunits)."""
        s = np.array(s, dtype=np.float64)
        self.L.orc_settime(_ptr(s))

    def units(self):
        """(temp0, temp0inv, kappa0) of the last compunits."""
        u = np.zeros(3)
        self.L.orc_get_units(_ptr(u))
        return u

    # -- chemistry (the CIE build: q of shape (nz, ny, nx, 12)) -------------
    def initchem(self, q):
        """initchem(q), chemistry.f90:26-70: fully neutral."""
        self.L.orc_initchem(_ptr(q))

    def chem_at(self, q, s):
        """chem(q) with the time scalars s (dt for the cooling)."""
        s = np.array(s, dtype=np.float64)
        self.L.orc_chem_at(_ptr(q), _ptr(s))

    def coef(self):
        """coef(13, 2) of compcoef as a (13, 2) array, and uv."""
        out = np.zeros(27)
        self.L.orc_get_coef(_ptr(out))
        return out[:26].reshape(13, 2), out[26]

    def peebles(self, s) -> float:
        """peebles(fpeebles), cosmology.f90:76-97, at the time scalars s."""
        s = np.array(s, dtype=np.float64)
        return float(self.L.orc_peebles(_ptr(s)))

    def expansion(self, q, s):
        """expansion(q), cosmology.f90:53-72, at the time scalars s."""
        s = np.array(s, dtype=np.float64)
        self.L.orc_expansion(_ptr(q), _ptr(s))

    # -- initial conditions -------------------------------------------------
    def ic_shocktube(self, dl, ul, pl, dr, ur, pr, x_diss, direction=1):
        q = self.zeros_q()
        rc = self.L.orc_ic_shocktube(_ptr(q), dl, ul, pl, dr, ur, pr, x_diss, int(direction))
        if rc:
            raise ValueError("bad shocktube direction")
        return q

    def ic_kh2d(self):
        q = self.zeros_q()
        self.L.orc_ic_kh2d(_ptr(q))
        return q

    def ic_kh3d(self, seed=42, amp=0.01):
        q = self.zeros_q()
        self.L.orc_ic_kh3d(_ptr(q), int(seed), float(amp))
        return q


def run_tube(task):
    """One 1D tube through the oracle's time loop (for a worker process of a
    spawned pool): task = (params dict, cells, q of shape (cells, 6)).
    Returns (q after the run, run info)."""
    kw, n, q = task
    o = Oracle(make_params(nx=n, ny=1, nz=1, **kw))
    o.set_threads(1)
    qq = np.ascontiguousarray(q, dtype=np.float64).reshape(1, 1, n, 6).copy()
    r = o.run(qq, 1 << 30)
    return qq.reshape(n, 6), r


def run_tubes(kw, lengths, q, workers=None):
    """Every tube of a packed batch (tubes concatenated, q of shape (cells,
    6)) through the oracle, longest first, in a spawned process pool (a
    broken worker raises instead of being restarted).  Returns a list of
    (q, info) in tube order."""
    import concurrent.futures as cf
    import multiprocessing as mp
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    tasks = [(kw, int(n), q[offs[i]:offs[i + 1]]) for i, n in enumerate(lengths)]
    order = sorted(range(len(tasks)), key=lambda i: -lengths[i])
    with cf.ProcessPoolExecutor(workers or os.cpu_count() or 4, mp_context=mp.get_context("spawn")) as pool:
        res = list(pool.map(run_tube, [tasks[i] for i in order], chunksize=4))
    out = [None] * len(tasks)
    for i, r in zip(order, res):
        out[i] = r
    return out
