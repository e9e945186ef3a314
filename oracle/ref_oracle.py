"""ctypes front end of oracle/_ref/libevora_ref.so -- TEST INFRASTRUCTURE ONLY.

libevora_ref.so is the reference's own Fortran hydro path translated
mechanically to C (oracle/ref/f2c.py) plus a harness that drives it like
main.f90 (oracle/ref/harness.c).  It pins the hand-written oracle
(evora_oracle.c) to the reference's sources.  The library is built here from
the sources under /root/reference (make -C oracle/ref); elsewhere the
prebuilt copy is used.  Same method names and array shapes as oracle.Oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .oracle import OracleParams, make_params  # noqa: F401  (re-exported for tests)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libevora_ref.so")
# the equilibrium-chemistry build (the reference compiled with -DCIE)
LIB_PATH_CIE = os.path.join(_HERE, "_ref", "libevora_ref_cie.so")
LIB_PATH_NCIE = os.path.join(_HERE, "_ref", "libevora_ref_ncie.so")
_PATHS = {False: LIB_PATH, True: LIB_PATH_CIE, "ncie": LIB_PATH_NCIE}
REF_SOURCES = "/root/reference/source"
_libs = {}
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def available() -> bool:
    return os.path.exists(LIB_PATH) or os.path.isdir(REF_SOURCES)


def lib(cie: bool = False):
    if cie not in _libs:
        if os.path.isdir(REF_SOURCES):
            subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref")], check=True)
        L = ctypes.CDLL(_PATHS[cie])
        L.ref_setup_c.argtypes = [ctypes.POINTER(OracleParams)]
        L.ref_sizes_c.argtypes = [ctypes.POINTER(ctypes.c_int64)] * 4
        L.ref_derived_c.argtypes = [_dp]
        L.ref_primitive_c.argtypes = [_dp, _dp]
        L.ref_bound_c.argtypes = [_dp]
        L.ref_hydrostep_c.argtypes = [_dp, _dp]
        L.ref_updatetime_c.argtypes = [_ip, _dp, _dp]
        L.ref_compevo_c.argtypes = [_dp, _dp, _dp, ctypes.c_double]
        L.ref_sweep_c.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_double]
        L.ref_run_c.argtypes = [_dp, ctypes.c_int, _dp, _ip, _dp, _ip]
        L.ref_ic_shocktube_c.argtypes = [_dp] + [ctypes.c_double] * 7 + [ctypes.c_int]
        L.ref_ic_kh_c.argtypes = [_dp]
        L.ref_riemann_c.argtypes = [_dp, _dp, _dp, ctypes.c_int]
        L.ref_thermalstep_c.argtypes = [_dp, _dp, _dp]
        L.ref_chem_c.argtypes = [_dp]
        L.ref_thermalconduction_c.argtypes = [_dp, _dp, ctypes.c_double]
        L.ref_coolstep_c.argtypes = [_dp, _dp, _dp]
        L.ref_run_trace_c.argtypes = [_dp, ctypes.c_int, _dp, _dp, _ip, _dp, _ip]
        L.ref_get_time_c.argtypes = [_dp]
        L.ref_get_units_c.argtypes = [_dp]
        L.ref_cosmostep_c.argtypes = [_dp]
        L.ref_compcosmo_c.argtypes = [_dp]
        L.ref_updatetime_cosmo_c.argtypes = [_ip, _ip, ctypes.c_int, _dp]
        L.ref_settime_c.argtypes = [_dp]
        L.ref_expansion_c.argtypes = [_dp, _dp]
        L.ref_peebles_c.argtypes = [_dp, _dp]
        L.ref_chem_at_c.argtypes = [_dp, _dp]
        L.ref_initchem_c.argtypes = [_dp]
        L.ref_get_coef_c.argtypes = [_dp]
        _libs[cie] = L
    return _libs[cie]


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class RefOracle:
    """The translated reference for one grid (module global state)."""

    def __init__(self, params: OracleParams | None = None, **kw):
        p_ = params if params is not None else make_params(**kw)
        chem = bool(getattr(p_, "chemistry", 0))
        self.L = lib(cie="ncie" if chem and getattr(p_, "noncie", 0) else chem)
        self.p = params if params is not None else make_params(**kw)
        if self.L.ref_setup_c(ctypes.byref(self.p)):
            raise ValueError("the reference stopped in compparameter/decomposition")
        d = np.zeros(16)
        self.L.ref_derived_c(_p(d))
        self.derived = dict(zip(["g", "g1", "g1inv", "gg1", "cfl", "de_thresh1", "dx", "dy", "dz",
                                 "dxinv", "dyinv", "dzinv", "x0", "y0", "z0", "volume"], d))

    @property
    def shape_q(self):
        return (self.p.nz, self.p.ny, self.p.nx, 12 if self.p.chemistry else 6)

    @property
    def nw(self):
        """Primitives per cell: 11 in the non-equilibrium build, else 5
        (global.f90:30-36)."""
        return 11 if (self.p.chemistry and self.p.noncie) else 5

    @property
    def shape_w(self):
        return (self.p.nz + 4, self.p.ny + 4, self.p.nx + 4, self.nw)

    @property
    def shape_evo(self):
        return (self.p.nz + 2, self.p.ny + 2, self.p.nx + 2, self.nw)

    @property
    def shape_s(self):
        return (self.p.nz + 2, self.p.ny + 2, self.p.nx + 2, 3, self.nw)

    def zeros_q(self):
        return np.zeros(self.shape_q)

    def primitive(self, w, q):
        return self.L.ref_primitive_c(_p(w), _p(q))

    def bound(self, w):
        return self.L.ref_bound_c(_p(w))

    def hydrostep(self, w, dt_in=1e99):
        d = ctypes.c_double(dt_in)
        st = self.L.ref_hydrostep_c(_p(w), ctypes.byref(d))
        return d.value, st

    def updatetime(self, t, dt):
        go = ctypes.c_int(1)
        tt, dd = ctypes.c_double(t), ctypes.c_double(dt)
        self.L.ref_updatetime_c(ctypes.byref(go), ctypes.byref(tt), ctypes.byref(dd))
        return bool(go.value), tt.value, dd.value

    def compevo(self, w, evo, s, dt):
        return self.L.ref_compevo_c(_p(w), _p(evo), _p(s), float(dt))

    def sweep(self, w, q, evo, s, dt):
        return self.L.ref_sweep_c(_p(w), _p(q), _p(evo), _p(s), float(dt))

    def thermalstep(self, q, w, dt_in=1e99):
        """thermalstep(q,w) (timestep.f90:72-104): min(dt_in, conduction limit)."""
        d = ctypes.c_double(dt_in)
        st = self.L.ref_thermalstep_c(_p(q), _p(w), ctypes.byref(d))
        return d.value, st

    def coolstep(self, q, w, dt_in=1e99):
        """coolstep(q,w) (timestep.f90:106-143), chemistry build: min(dt_in,
        cooling limit); writes the abundances back into q as there."""
        d = ctypes.c_double(dt_in)
        st = self.L.ref_coolstep_c(_p(q), _p(w), ctypes.byref(d))
        return d.value, st

    def chem(self, q):
        """chem(q) (chemistry.f90:72-121), plain build: the pressure floors."""
        return self.L.ref_chem_c(_p(q))

    def thermalconduction(self, q, w, dt):
        """thermalconduction(q,w) (conduction.f90:26-122) over dt."""
        return self.L.ref_thermalconduction_c(_p(q), _p(w), float(dt))

    def riemann(self, wl, wr, direction):
        wl = np.ascontiguousarray(wl, dtype=np.float64)
        wr = np.ascontiguousarray(wr, dtype=np.float64)
        f = np.zeros(6)
        st = self.L.ref_riemann_c(_p(wl), _p(wr), _p(f), int(direction))
        return f, st

    def run(self, q, max_steps, trace=False):
        t, dt = ctypes.c_double(), ctypes.c_double()
        steps, go = ctypes.c_int(), ctypes.c_int()
        tr = np.zeros((max(int(max_steps), 1), 8)) if trace else None
        st = self.L.ref_run_trace_c(_p(q), int(max_steps), _p(tr) if trace else None, ctypes.byref(t),
                                    ctypes.byref(steps), ctypes.byref(dt), ctypes.byref(go))
        out = dict(t=t.value, steps=steps.value, dt=dt.value, go=bool(go.value), stopped=int(st))
        if trace:
            out["trace"] = tr[:steps.value].copy()
        return out

    # -- comoving time scalars (t, dt, cosmo, oldcosmo, cosmodot, expand, redshift)
    def time(self):
        s = np.zeros(7)
        self.L.ref_get_time_c(_p(s))
        return s

    def units(self):
        """(temp0, temp0inv, kappa0) of module global."""
        u = np.zeros(3)
        self.L.ref_get_units_c(_p(u))
        return u

    def cosmostep(self, s):
        s = np.array(s, dtype=np.float64)
        st = self.L.ref_cosmostep_c(_p(s))
        return s, st

    def compcosmo(self, s):
        s = np.array(s, dtype=np.float64)
        st = self.L.ref_compcosmo_c(_p(s))
        return s, st

    def updatetime_cosmo(self, go, s, k=1):
        s = np.array(s, dtype=np.float64)
        g, d = ctypes.c_int(1 if go else 0), ctypes.c_int(0)
        st = self.L.ref_updatetime_cosmo_c(ctypes.byref(g), ctypes.byref(d), int(k), _p(s))
        return bool(g.value), bool(d.value), s, st

    def settime(self, s):
        """Sets the time scalars and runs compunits."""
        s = np.array(s, dtype=np.float64)
        return self.L.ref_settime_c(_p(s))

    def peebles(self, s):
        s = np.array(s, dtype=np.float64)
        f = ctypes.c_double()
        st = self.L.ref_peebles_c(_p(s), ctypes.byref(f))
        return f.value, st

    def expansion(self, q, s):
        s = np.array(s, dtype=np.float64)
        return self.L.ref_expansion_c(_p(q), _p(s))

    # -- chemistry (the CIE build: q of shape (nz, ny, nx, 12)) -------------
    def initchem(self, q):
        return self.L.ref_initchem_c(_p(q))

    def chem_at(self, q, s):
        """chem(q) with the time scalars s (dt for the cooling)."""
        s = np.array(s, dtype=np.float64)
        return self.L.ref_chem_at_c(_p(q), _p(s))

    def coef(self):
        """coef(13, 2) as a (13, 2) array, and uv."""
        out = np.zeros(27)
        self.L.ref_get_coef_c(_p(out))
        return out[:26].reshape(13, 2), out[26]

    def ic_shocktube(self, dl, ul, pl, dr, ur, pr, x_diss, direction=1):
        q = self.zeros_q()
        if self.L.ref_ic_shocktube_c(_p(q), dl, ul, pl, dr, ur, pr, x_diss, int(direction)):
            raise ValueError("the reference stopped in ic")
        return q

    def ic_kh2d(self):
        q = self.zeros_q()
        self.L.ref_ic_kh_c(_p(q))
        return q
