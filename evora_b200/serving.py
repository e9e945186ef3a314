"""Request loop with continuous batching over the C ABI (evora_server_*).

A request is an initial state in the reference layout q (nz, ny, nx, 6), its
grid size and an end time.  `Server.tick()` admits pending requests while
their device footprint fits the HBM budget, advances every admitted request
by up to `steps_per_tick` steps (1D tubes together in one persistent
launch, 2D/3D grids concurrently on their own streams) and retires finished
ones.  Latency is the time from submit to the read-back of the result."""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import EvoraParams, check, lib
from .hydro import FP32

PENDING, RUNNING, DONE, FAILED = 0, 1, 2, 3


class Server:
    def __init__(self, base: EvoraParams, precision: int = FP32, flags: int = 0, hbm_budget_bytes: float = 150e9,
                 steps_per_tick: int = 64, max_tube_cells: int = 8192, max_tubes: int = 4096):
        h = ctypes.c_void_p()
        check(lib().evora_server_create(ctypes.byref(base), precision, flags, float(hbm_budget_bytes),
                                        steps_per_tick, max_tube_cells, max_tubes, ctypes.byref(h)),
              "server_create")
        self._h = h
        self.shapes = {}
        self._borrowed = {}   # id -> (q0, out) arrays the server reads / writes after submit

    def close(self):
        if getattr(self, "_h", None):
            lib().evora_server_destroy(self._h)
            self._h = None
        self._borrowed = {}

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, q0: np.ndarray, tend: float, boundtype: int = 0) -> int:
        """q0: (nz, ny, nx, 6) float64 (a 1D tube may be given as (n, 6));
        boundtype 1..3 overrides the server's for this request."""
        q0 = np.ascontiguousarray(q0, dtype=np.float64)
        if q0.ndim == 2:
            nz, ny, nx = 1, 1, q0.shape[0]
        else:
            nz, ny, nx = q0.shape[:3]
        rid = ctypes.c_int64()
        check(lib().evora_server_submit(self._h, nx, ny, nz, float(tend), int(boundtype),
                                        ctypes.c_void_p(q0.ctypes.data), ctypes.byref(rid)), "server_submit")
        self.shapes[rid.value] = q0.shape
        return rid.value

    def submit_borrowed(self, q0: np.ndarray, tend: float, boundtype: int = 0, out=None) -> int:
        """As submit(), but the server's copy threads read q0 after the call
        and, with `out` (float64, C-contiguous, q0's shape), write the result
        into it before the request reports done, so the host copies overlap
        the device's rounds.  The server keeps both arrays referenced until
        result() delivers the request."""
        q0 = np.ascontiguousarray(q0, dtype=np.float64)
        if q0.ndim == 2:
            nz, ny, nx = 1, 1, q0.shape[0]
        else:
            nz, ny, nx = q0.shape[:3]
        if out is not None and (out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]
                                or out.shape != q0.shape):
            raise ValueError("out must be a C-contiguous float64 array of q0's shape")
        rid = ctypes.c_int64()
        check(lib().evora_server_submit_borrowed(self._h, nx, ny, nz, float(tend), int(boundtype),
                                                 ctypes.c_void_p(q0.ctypes.data),
                                                 None if out is None else ctypes.c_void_p(out.ctypes.data),
                                                 ctypes.byref(rid)), "server_submit_borrowed")
        self.shapes[rid.value] = q0.shape
        self._borrowed[rid.value] = (q0, out)
        return rid.value

    def tick(self):
        a, p = ctypes.c_int32(), ctypes.c_int32()
        check(lib().evora_server_tick(self._h, ctypes.byref(a), ctypes.byref(p)), "server_tick")
        return a.value, p.value

    def state(self, rid: int) -> int:
        st = ctypes.c_int32()
        lib().evora_server_result(self._h, int(rid), None, None, None, ctypes.byref(st))
        return st.value

    def result(self, rid: int, out=None):
        """(q, latency_s, steps, err) for a finished request, else None.  q
        is written into `out` when given (float64, C-contiguous, the
        request's shape), else into a new array."""
        st = self.state(rid)
        if st not in (DONE, FAILED):
            return None
        if out is None and rid in self._borrowed:
            out = self._borrowed[rid][1]
        if out is not None:
            if out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"] or out.shape != tuple(self.shapes[rid]):
                raise ValueError("out must be a C-contiguous float64 array of the request's shape")
            q = out
        else:
            q = np.empty(self.shapes[rid])
        lat, steps, st2 = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int32()
        err = lib().evora_server_result(self._h, int(rid), ctypes.c_void_p(q.ctypes.data), ctypes.byref(lat),
                                        ctypes.byref(steps), ctypes.byref(st2))
        del self.shapes[rid]
        self._borrowed.pop(rid, None)
        return q, lat.value, steps.value, int(err)

    def stats(self):
        p50, p99, span = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        done, cu = ctypes.c_int64(), ctypes.c_int64()
        check(lib().evora_server_stats(self._h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(done),
                                       ctypes.byref(cu), ctypes.byref(span)), "server_stats")
        return dict(p50_s=p50.value, p99_s=p99.value, completed=done.value, cell_updates=cu.value,
                    span_s=span.value)

    def completed(self, max_ids: int = 4096):
        """Ids finished since the last call (oldest first)."""
        buf = (ctypes.c_int64 * max_ids)()
        n = ctypes.c_int32()
        check(lib().evora_server_completed(self._h, buf, max_ids, ctypes.byref(n)), "server_completed")
        return list(buf[:n.value])

    def profile(self):
        """Host seconds per round phase, the number of rounds, and the device
        seconds of the rounds' tube launches and multi-grid steps."""
        out = (ctypes.c_double * 7)()
        check(lib().evora_server_profile(self._h, out), "server_profile")
        names = ["launch", "readback", "admission", "wait", "free", "detect"]
        d = {n: out[i] for i, n in enumerate(names)}
        d["rounds"] = int(out[6])
        tm, bm = ctypes.c_double(), ctypes.c_double()
        check(lib().evora_server_device_ms(self._h, ctypes.byref(tm), ctypes.byref(bm)), "server_device_ms")
        d["device_tubes"] = 1e-3 * tm.value
        d["device_batch"] = 1e-3 * bm.value
        return d
