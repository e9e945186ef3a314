"""Python front end of the evora hydro update on B200.

Mirrors the reference's operator interface for the hydro path: the drop-in
routines `primitive`, `bound`, `hydrostep`, `updatetime`, `compevo`, `sweep`
(same names, arguments and array layouts as muscl.f90 / boundary.f90 /
timestep.f90), and the resident `Grid` that advances whole steps on the
device.  Arrays are numpy (host) or torch CUDA tensors (device), float64,
C-contiguous, in the reference's column-major layouts read in C order:

    q   (nz, ny, nx, 6)           q(6, nx, ny, nz)                  main.f90:72
    w   (nz+4, ny+4, nx+4, 5)     w(5, -1:nx+2, -1:ny+2, -1:nz+2)   main.f90:73
    evo (nz+2, ny+2, nx+2, 5)     evo(5, 0:nx+1, ...)               main.f90:74
    s   (nz+2, ny+2, nx+2, 3, 5)  s(5, 3, 0:nx+1, ...)              main.f90:75

Every call goes through libevora_b200.so; errors raise EvoraError with the
reference condition that caused them.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import NDUMP, EvoraDerived, EvoraError, EvoraParams, EvoraTime, check, lib

FP64 = 0
FP32 = 1
CARRY_ENTROPY = 1
STRICT = 2
REFERENCE_KERNELS = 4
# tile entry of the FP32 table that runs two cells per thread on packed FP32
# pairs (its sums are associated differently from the other FP32 kernels)
FP32_PAIR_TILE = 5   # EVORA_FP32_PAIR_TILE
# resident modes of the drop-in layer (evora_set_resident)
RESIDENT_FP64 = 1
RESIDENT_FP32 = 2


# ------------------------------------------------------------- parameters --
def default_params(**overrides) -> EvoraParams:
    """readparameter defaults (parameter.f90:41-82), then keyword overrides.
    dump_redshift takes a sequence (the rest stays -1, parameter.f90:82)."""
    p = EvoraParams()
    lib().evora_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"unknown parameter {k!r}")
        if k == "dump_redshift":
            v = list(v)
            if len(v) > NDUMP:
                raise ValueError(f"at most {NDUMP} dump redshifts")
            for i in range(NDUMP):
                p.dump_redshift[i] = float(v[i]) if i < len(v) else -1.0
            continue
        setattr(p, k, v)
    return p


def _time(s) -> EvoraTime:
    if isinstance(s, EvoraTime):
        return s
    t = EvoraTime()
    for k, v in dict(s).items():
        setattr(t, k, float(v))
    return t


def derived(p: EvoraParams) -> EvoraDerived:
    """compparameter (parameter.f90:164-265)."""
    d = EvoraDerived()
    check(lib().evora_compparameter(ctypes.byref(p), ctypes.byref(d)), "compparameter")
    return d


def shapes(p: EvoraParams):
    """C shapes of the reference arrays: q has 12 values per cell with
    chemistry (q(7:12) = the species), else 6; w has 11 primitives in the
    non-equilibrium build (noncie), else 5."""
    nx, ny, nz = p.nx, p.ny, p.nz
    nq = 12 if p.chemistry else 6
    nw = 11 if p.chemistry and p.noncie else 5
    return dict(q=(nz, ny, nx, nq), w=(nz + 4, ny + 4, nx + 4, nw),
                evo=(nz + 2, ny + 2, nx + 2, nw), s=(nz + 2, ny + 2, nx + 2, 3, nw))


def _ptr(a, shape=None, writable=True):
    """Address of a float64 C-contiguous numpy array or torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise TypeError("arrays must be float64 and C-contiguous")
        if writable and not a.flags["WRITEABLE"]:
            raise TypeError("array is read-only")
        if shape is not None and a.shape != tuple(shape):
            raise ValueError(f"shape {a.shape} != expected {tuple(shape)}")
        return ctypes.c_void_p(a.ctypes.data)
    try:
        import torch
    except ImportError:  # pragma: no cover
        raise TypeError("unsupported array type")
    if isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("tensors must be float64 and contiguous")
        if shape is not None and tuple(a.shape) != tuple(shape):
            raise ValueError(f"shape {tuple(a.shape)} != expected {tuple(shape)}")
        return ctypes.c_void_p(a.data_ptr())
    raise TypeError("unsupported array type")


# ----------------------------------------------------------- drop-in layer --
class DropIn:
    """The drop-in routines for one set of module-global parameters."""

    def __init__(self, params: EvoraParams, strict: bool = False):
        self.params = params
        self.shape = shapes(params)
        check(lib().evora_set_params(ctypes.byref(params)), "set_params")
        check(lib().evora_set_strict(1 if strict else 0), "set_strict")

    def _activate(self):
        check(lib().evora_set_params(ctypes.byref(self.params)), "set_params")

    def set_resident(self, mode: int):
        """Resident mode (RESIDENT_FP64, RESIDENT_FP32, or 0 to end it): the
        routines keep the state on the GPU between calls; host q is brought
        up to date by sync(q) (see evora_set_resident)."""
        check(lib().evora_set_resident(int(mode)), "set_resident")

    def sync(self, q):
        """Copies the resident state back into host array q."""
        check(lib().evora_sync(_ptr(q, self.shape["q"])), "sync")

    def invalidate(self, q):
        """The caller changed host q: the next primitive uploads it again."""
        check(lib().evora_invalidate(_ptr(q, self.shape["q"], False)), "invalidate")

    def primitive(self, w, q):
        """primitive(w,q), muscl.f90:26-43."""
        check(lib().evora_primitive(_ptr(w, self.shape["w"]), _ptr(q, self.shape["q"])), "primitive")

    def bound(self, w):
        """bound(w), boundary.f90:26-113."""
        check(lib().evora_bound(_ptr(w, self.shape["w"])), "bound")

    def hydrostep(self, w, dt: float = 1e99) -> float:
        """hydrostep(w), timestep.f90:26-57; returns min(cfl*v, dt)."""
        d = ctypes.c_double(dt)
        check(lib().evora_hydrostep(_ptr(w, self.shape["w"], False), ctypes.byref(d)), "hydrostep")
        return d.value

    def updatetime(self, go: bool, t: float, dt: float, k: int = 1):
        """updatetime(go,dump,k), timestep.f90:147-171; returns (go, t, dt)."""
        g = ctypes.c_int32(1 if go else 0)
        dump = ctypes.c_int32(0)
        kk = ctypes.c_int32(k)
        tt, dd = ctypes.c_double(t), ctypes.c_double(dt)
        check(lib().evora_updatetime(ctypes.byref(g), ctypes.byref(dump), ctypes.byref(kk),
                                     ctypes.byref(tt), ctypes.byref(dd)), "updatetime")
        return bool(g.value), tt.value, dd.value

    def compevo(self, w, evo, s, dt: float):
        """compevo(w,evo,s), muscl.f90:45-113."""
        check(lib().evora_compevo(_ptr(w, self.shape["w"], False), _ptr(evo, self.shape["evo"]),
                                  _ptr(s, self.shape["s"]), float(dt)), "compevo")

    def sweep(self, w, q, evo, s, dt: float):
        """sweep(w,q,evo,s), muscl.f90:171-274."""
        check(lib().evora_sweep(_ptr(w, self.shape["w"], False), _ptr(q, self.shape["q"]),
                                _ptr(evo, self.shape["evo"], False), _ptr(s, self.shape["s"], False),
                                float(dt)), "sweep")

    def _phi_ptr(self, phi):
        if not isinstance(phi, np.ndarray) or phi.dtype != np.complex128 or not phi.flags["C_CONTIGUOUS"]:
            raise TypeError("phi must be a C-contiguous complex128 array")
        if phi.shape != tuple(self.shape["q"][:3]):
            raise ValueError(f"phi shape {phi.shape} != {tuple(self.shape['q'][:3])}")
        return ctypes.c_void_p(phi.ctypes.data)

    def gravpotential(self, q, phi):
        """gravpotential(q,phi), gravitation.f90:26-53 (non-comoving): phi is
        complex(8) phi(nx,ny,nz), C shape (nz, ny, nx) complex128; its
        imaginary part is written as 0."""
        check(lib().evora_gravpotential(_ptr(q, self.shape["q"], False), self._phi_ptr(phi)), "gravpotential")

    def chem(self, q):
        """chem(q), chemistry.f90:72-121: pressure(), with chemistry the CIE
        species and the cooling over the dt of settime, and the temperature /
        Jeans pressure floors."""
        check(lib().evora_chem(_ptr(q, self.shape["q"])), "chem")

    def initchem(self, q):
        """initchem(q), chemistry.f90:26-70, on a host q (nz, ny, nx, 12):
        fully neutral species."""
        check(lib().evora_initchem(_ptr(q, self.shape["q"])), "initchem")

    def thermalstep(self, q, w, dt: float = 1e99) -> float:
        """thermalstep(q,w), timestep.f90:72-104: min(dt, conduction limit);
        q is resynchronised in place with dual energy, as in the reference."""
        d = ctypes.c_double(dt)
        check(lib().evora_thermalstep(_ptr(q, self.shape["q"]), _ptr(w, self.shape["w"], False),
                                      ctypes.byref(d)), "thermalstep")
        return d.value

    def coolstep(self, q, w, dt: float = 1e99) -> float:
        """coolstep(q,w), timestep.f90:106-143: min(dt, c_cooldt times the
        smallest cooling time).  As in the reference, q(7:12) is overwritten
        with the equilibrium abundances at the nH, nHe the last chem or
        initchem left (its last cell's)."""
        d = ctypes.c_double(dt)
        check(lib().evora_coolstep(_ptr(q, self.shape["q"]), _ptr(w, self.shape["w"], False),
                                   ctypes.byref(d)), "coolstep")
        return d.value

    def thermalconduction(self, q, w, dt: float):
        """thermalconduction(q,w), conduction.f90:26-122 (simplekappa)."""
        check(lib().evora_thermalconduction(_ptr(q, self.shape["q"]), _ptr(w, self.shape["w"], False),
                                            float(dt)), "thermalconduction")

    def gravintegration(self, q, phi, dt: float):
        """gravintegration(q,phi,...), gravitation.f90:170-243 (one process,
        so no boundary buffers): the gravitational source terms over dt."""
        check(lib().evora_gravintegration(_ptr(q, self.shape["q"]), self._phi_ptr(phi), float(dt)),
              "gravintegration")

    # comoving time scalars: dicts with the fields of evora_time
    def cosmostart(self) -> dict:
        """cosmostart (cosmology.f90:26-36) after compparameter: the time
        scalars at the start of the run."""
        s = EvoraTime()
        check(lib().evora_cosmostart(ctypes.byref(s)), "cosmostart")
        return s.as_dict()

    def cosmostep(self, s) -> dict:
        """cosmostep (timestep.f90:59-70): dt = min(a / (da/dt) c_cosmo, dt)."""
        t = _time(s)
        check(lib().evora_cosmostep(ctypes.byref(t)), "cosmostep")
        return t.as_dict()

    def compcosmo(self, s) -> dict:
        """compcosmo (cosmology.f90:38-51): a advanced over dt."""
        t = _time(s)
        check(lib().evora_compcosmo(ctypes.byref(t)), "compcosmo")
        return t.as_dict()

    def updatetime_cosmo(self, go: bool, s, k: int = 1):
        """updatetime(go,dump,k), timestep.f90:147-171, both branches;
        returns (go, dump, time scalars)."""
        t = _time(s)
        g, d, kk = ctypes.c_int32(1 if go else 0), ctypes.c_int32(0), ctypes.c_int32(k)
        check(lib().evora_updatetime_cosmo(ctypes.byref(g), ctypes.byref(d), ctypes.byref(kk),
                                           ctypes.byref(t)), "updatetime")
        return bool(g.value), bool(d.value), t.as_dict()

    def peebles(self, s) -> float:
        """peebles(fpeebles), cosmology.f90:76-97: d ln D / d ln a at s's a."""
        f = ctypes.c_double()
        check(lib().evora_peebles(ctypes.byref(_time(s)), ctypes.byref(f)), "peebles")
        return f.value

    def settime(self, s):
        """The time scalars the routines read from module global (dt and
        expand for expansion, a for the comoving gravity source and the
        comoving units)."""
        check(lib().evora_settime(ctypes.byref(_time(s))), "settime")

    def expansion(self, q):
        """expansion(q), cosmology.f90:53-72, with dt and expand of settime."""
        check(lib().evora_expansion(_ptr(q, self.shape["q"])), "expansion")


# ---------------------------------------------------------- resident grid --
class Grid:
    """A grid whose state stays on the current CUDA device across steps."""

    def __init__(self, params: EvoraParams, precision: int = FP64, flags: int = 0, stream=None):
        self.params = params
        self.precision = precision
        self.flags = flags
        self.shape_q = shapes(params)["q"]
        h = ctypes.c_void_p()
        check(lib().evora_grid_create(ctypes.byref(params), precision, flags, ctypes.byref(h)),
              "grid_create")
        self._h = h
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "_h", None):
            lib().evora_grid_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream or a raw cudaStream_t integer."""
        raw = getattr(stream, "cuda_stream", stream)
        check(lib().evora_grid_set_stream(self._h, ctypes.c_void_p(int(raw))), "grid_set_stream")

    def set_q(self, q):
        check(lib().evora_grid_set_q(self._h, _ptr(q, self.shape_q, False)), "grid_set_q")

    def get_q(self, out=None):
        if out is None:
            out = np.empty(self.shape_q)
        check(lib().evora_grid_get_q(self._h, _ptr(out, self.shape_q)), "grid_get_q")
        return out

    def step(self, nsteps: int = 1, sync: bool = True):
        st = lib().evora_grid_step(self._h, int(nsteps), 1 if sync else 0)
        check(st, "grid_step")

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        go, k = ctypes.c_int32(), ctypes.c_int64()
        check(lib().evora_grid_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(go),
                                    ctypes.byref(k)), "grid_time")
        return dict(t=t.value, dt=dt.value, go=bool(go.value), k=k.value)

    def status(self) -> int:
        return int(lib().evora_grid_status(self._h))

    def totals(self):
        out = (ctypes.c_double * 6)()
        check(lib().evora_grid_totals(self._h, out), "grid_totals")
        return np.array(out[:])

    def autotune(self, reps: int = 3):
        """Times every tile shape of the fused kernel on this grid, keeps the
        fastest; returns (chosen index, ms per launch for each shape)."""
        chosen = ctypes.c_int32()
        ms = (ctypes.c_double * 16)()
        check(lib().evora_grid_autotune(self._h, int(reps), ctypes.byref(chosen), ms, 16), "grid_autotune")
        return chosen.value, [v for v in ms[:16] if v > 0]

    def set_tile(self, tile: int):
        check(lib().evora_grid_set_tile(self._h, int(tile)), "grid_set_tile")

    def set_timing(self, on: bool = True):
        check(lib().evora_grid_set_timing(self._h, 1 if on else 0), "grid_set_timing")

    def timing(self):
        """Summed event times since timing was switched on: update_ms is the
        update and the physics after it (fused_ms and physics_ms apart)."""
        cf, up, ph = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n, la = ctypes.c_int64(), ctypes.c_int64()
        check(lib().evora_grid_timing_split(self._h, ctypes.byref(cf), ctypes.byref(up), ctypes.byref(ph),
                                            ctypes.byref(n), ctypes.byref(la)), "grid_timing")
        return dict(update_ms=up.value + ph.value, fused_ms=up.value, physics_ms=ph.value, cfl_ms=cf.value,
                    steps=n.value, launches=la.value)

    def cosmo(self):
        """The time scalars and the pending dump: (dict, k) with k the
        dump_redshift index whose dump the last step raised (0: none).  A
        pending dump holds the grid; this call clears it."""
        s, d = EvoraTime(), ctypes.c_int32()
        check(lib().evora_grid_cosmo(self._h, ctypes.byref(s), ctypes.byref(d)), "grid_cosmo")
        return s.as_dict(), d.value

    def run(self, max_steps: int = 1 << 30, chunk: int = 64, on_dump=None):
        """Advances until updatetime clears go (or max_steps).  With
        comoving dumps the grid stops at each one: on_dump(grid, k) is called
        there (the state is the dump's), then the run goes on."""
        k_start = self.time()["k"]
        done = 0
        while done < max_steps:
            self.step(min(chunk, max_steps - done), sync=True)
            if self.params.supercomoving:
                _, dump = self.cosmo()
                if dump and on_dump is not None:
                    on_dump(self, dump)
            tm = self.time()
            done = tm["k"] - k_start   # steps taken (held ones do not count)
            if not tm["go"]:
                break
        return self.time()


class MultiGrid:
    """Resident 2D and 3D grids of uneven sizes advanced together: per step
    one control kernel, one persistent update launch over the tiles of all
    member grids, one closing control kernel (evora_multigrid_*)."""

    def __init__(self, precision: int = FP32, flags: int = 0, stream=None):
        h = ctypes.c_void_p()
        raw = getattr(stream, "cuda_stream", stream) if stream is not None else None
        check(lib().evora_multigrid_create(precision, flags, ctypes.c_void_p(int(raw) if raw else 0),
                                           ctypes.byref(h)), "multigrid_create")
        self._h = h
        self.members = []

    def close(self):
        if getattr(self, "_h", None):
            lib().evora_multigrid_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, grid: "Grid"):
        check(lib().evora_multigrid_add(self._h, grid._h), "multigrid_add")
        self.members.append(grid)

    def remove(self, grid: "Grid"):
        check(lib().evora_multigrid_remove(self._h, grid._h), "multigrid_remove")
        self.members.remove(grid)

    def step(self, nsteps: int = 1, sync: bool = True):
        check(lib().evora_multigrid_step(self._h, int(nsteps), 1 if sync else 0), "multigrid_step")

    def status(self):
        """[(go, err, k)] in member order (waits for the batch)."""
        n = len(self.members)
        go = (ctypes.c_int32 * max(n, 1))()
        err = (ctypes.c_uint32 * max(n, 1))()
        k = (ctypes.c_int64 * max(n, 1))()
        cnt = ctypes.c_int32()
        check(lib().evora_multigrid_status(self._h, None, go, err, k, n, ctypes.byref(cnt)), "multigrid_status")
        return [(bool(go[i]), int(err[i]), int(k[i])) for i in range(cnt.value)]


__all__ = ["EvoraError", "EvoraParams", "EvoraDerived", "default_params", "derived", "shapes",
           "DropIn", "Grid", "Batch", "FP64", "FP32", "CARRY_ENTROPY", "STRICT", "REFERENCE_KERNELS",
           "FP32_PAIR_TILE", "RESIDENT_FP64", "RESIDENT_FP32", "MultiGrid"]


# --------------------------------------------------------- batched tubes --
class Batch:
    """Independent 1D tubes advanced together (evora_batch_*): each tube is a
    run of the reference loop on its own grid of n[i] cells, with its own
    time and end time."""

    def __init__(self, params: EvoraParams, lengths, precision: int = FP32, flags: int = 0):
        self.params = params
        self.n = [int(x) for x in lengths]
        self.offsets = np.concatenate([[0], np.cumsum(self.n)]).astype(np.int64)
        arr = (ctypes.c_int32 * len(self.n))(*self.n)
        h = ctypes.c_void_p()
        check(lib().evora_batch_create(ctypes.byref(params), len(self.n), arr, precision, flags,
                                       ctypes.byref(h)), "batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().evora_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_q(self, q, tube: int = -1):
        """q: (n[tube], 6) for one tube, or (sum n, 6) for all (tube = -1)."""
        cells = sum(self.n) if tube < 0 else self.n[tube]
        check(lib().evora_batch_set_q(self._h, tube, _ptr(q, (cells, 6), False)), "batch_set_q")

    def get_q(self, tube: int = -1, out=None):
        cells = sum(self.n) if tube < 0 else self.n[tube]
        if out is None:
            out = np.empty((cells, 6))
        check(lib().evora_batch_get_q(self._h, tube, _ptr(out, (cells, 6))), "batch_get_q")
        return out

    def set_stream(self, stream):
        """stream: a (non-default) torch.cuda.Stream or raw cudaStream_t."""
        raw = getattr(stream, "cuda_stream", stream)
        check(lib().evora_batch_set_stream(self._h, ctypes.c_void_p(int(raw))), "batch_set_stream")

    def set_tend(self, tube: int, tend: float):
        check(lib().evora_batch_set_tend(self._h, tube, float(tend)), "batch_set_tend")

    def run(self, max_steps: int = 0, sync: bool = True):
        """Advances every running tube; returns the OR of tube errors (sync)."""
        return int(lib().evora_batch_run(self._h, int(max_steps), 1 if sync else 0))

    def info(self, tube: int):
        t, dt = ctypes.c_double(), ctypes.c_double()
        go, st = ctypes.c_int32(), ctypes.c_int32()
        k = ctypes.c_int64()
        err = lib().evora_batch_info(self._h, tube, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(go),
                                     ctypes.byref(k), ctypes.byref(st))
        return dict(t=t.value, dt=dt.value, go=bool(go.value), k=k.value, status=st.value, err=int(err))

    def cell_updates(self) -> int:
        v = ctypes.c_int64()
        check(lib().evora_batch_steps_done(self._h, ctypes.byref(v)), "batch_steps_done")
        return v.value

    def configure(self, threads: int = 256, ctas_per_sm: int = 2):
        check(lib().evora_batch_configure(self._h, threads, ctas_per_sm), "batch_configure")

    def autotune_batch(self, steps: int = 20):
        return self.autotune(steps)

    def autotune(self, steps: int = 20):
        th, ct = ctypes.c_int32(), ctypes.c_int32()
        check(lib().evora_batch_autotune(self._h, int(steps), ctypes.byref(th), ctypes.byref(ct)), "batch_autotune")
        return th.value, ct.value
