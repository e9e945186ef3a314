"""Benchmark of the evora hydro update on B200.

Workload (one "step" = one full hydro step of main.f90:109-155: primitive,
ghost fill, CFL reduction, updatetime, predictor, three sweeps): the 3D
Kelvin-Helmholtz instability on a 256^3 periodic grid, gamma = 5/3, HLLC,
minmod, CFL 0.5 (the reference's default, parameter.f90:46), seeded vy
perturbation (SplitMix64 seed 42, amplitude 0.01, modes k = 1..4), synthetic
IC built on the host in FP64.

Headline `value`: the FP32 form (FP32 state/slopes/fluxes, FP64 pressure
recovery where kin > E/2, FP64 CFL reduction) in cell-updates/s, inputs
resident in HBM.  The FP64 form is measured on the same workload and
reported under "fp64", with the relative L1 density error of FP32 vs FP64
after the same steps.  `e2e` is the same metric through the public C ABI
with host buffers: every step uploads q(6,256,256,256) from pinned host
memory, advances one step and reads q back.

`--impl reference` times the CPU oracle (the C restatement of the
reference's hot path; the reference is Fortran and no Fortran compiler exists
on this image) on all host threads, on a bounded z-slab sample of the same
workload.

Multi-GPU: the single-grid path has no exchange (one grid per GPU, no domain
decomposition), so N > 1 runs N independent replicas, one per rank
("scaling": "weak"); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = NZ = 256
AUTOTUNE = True
TILES = None       # (fp32 tile, fp64 tile) pinned by --tiles
CHEMISTRY = True   # the cosmological box runs the CIE chemistry and cooling
GAMMA = 5.0 / 3.0
CFL = 0.5
METRIC = "cell-updates/s"
BYTES_PER_CELL = {"f32": 40, "f64": 80}   # 5 fields read + written once
WORKLOAD = "3D Kelvin-Helmholtz 256^3 periodic, gamma=5/3, HLLC, minmod, CFL 0.5"


def kh_params(ev, nz=None, gravity=0, conduction=0, box=1.0, **extra):
    return ev.default_params(nx=NX, ny=NY, nz=nz or NZ, g=GAMMA, cfl=CFL, boundtype=2, solver=2,
                             limiter=1, tend=1.0e6, gravity=gravity, conduction=conduction,
                             simplekappa=conduction, xmax=box, ymax=box, zmax=box, **extra)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch from a committed ncu summary (profiles/*.md):
    a line 'traffic_bytes_per_launch: N'."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"evora_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def wait_first_sample(self, timeout=3.0):
        """Blocks until nvidia-smi has written its first sample."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout:
            self.f.flush()
            if os.path.exists(self.path) and os.path.getsize(self.path) > 0:
                return
            time.sleep(0.05)

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pick_tile(g, precision):
    """The tile shape of the fused kernel: --tiles pins it (profiling runs
    reproduce the shape a timed run chose), else autotune, else the default."""
    import evora_b200 as ev
    if TILES is not None:
        t = TILES[0 if precision == ev.FP32 else 1]
        g.set_tile(t)
        return t, []
    return g.autotune(reps=3) if AUTOTUNE else (0, [])


def time_grid(ev, torch, q, precision, steps, warmup, stream, gravity=0, conduction=0, box=1.0, **extra):
    """Device-timed resident steps; returns (ms_total, kernel timing, grid)."""
    g = ev.Grid(kh_params(ev, gravity=gravity, conduction=conduction, box=box, **extra), precision)
    g.set_stream(stream)
    g.set_q(q)
    g.tuning = pick_tile(g, precision)
    g.step(warmup, sync=True)
    torch.cuda.synchronize()
    g.set_timing(True)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    g.step(steps, sync=False)
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    kt = g.timing()
    st = g.status()
    if st:
        raise RuntimeError(f"grid status {st}")
    return ms, kt, g


def time_e2e(ev, torch, q_pinned, outs_pinned, precision, steps):
    """The step through the public API with host buffers: every step uploads
    q(6, nx, ny, nz) (FP64, pinned host) with set_q, advances it one step and
    reads it back with get_q.  Two grids on two streams, each driven by its
    own host thread, alternate the steps, so one grid's upload overlaps the
    other's download (PCIe is full duplex) and the kernels.  Returns the wall
    time of all `steps` steps."""
    import threading
    k = len(outs_pinned)
    grids = [ev.Grid(kh_params(ev), precision) for _ in range(k)]
    streams = [torch.cuda.Stream() for _ in range(k)]
    for g, st, out in zip(grids, streams, outs_pinned):
        g.set_stream(st)
        g.set_q(q_pinned)
        g.step(1)
        g.get_q(out)
    torch.cuda.synchronize()
    share = [steps // k + (1 if i < steps % k else 0) for i in range(k)]
    errors = []

    def work(i):
        try:
            for _ in range(share[i]):
                grids[i].set_q(q_pinned)
                grids[i].step(1, sync=True)
                grids[i].get_q(outs_pinned[i])
        except Exception as e:  # reported after the join
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(k)]
    t0 = time.perf_counter()
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    el = time.perf_counter() - t0
    for g in grids:
        g.close()
    if errors:
        raise errors[0]
    return el


def time_dropin_resident(ev, q, mode, steps, warmup):
    """main.f90:109-155's call order (primitive, bound, hydrostep,
    updatetime, compevo, sweep) through the drop-in C ABI on host arrays, in
    resident mode: the state stays on the GPU between the calls, and
    evora_sync brings q back once at the end.  Returns (ms per step of the
    loop, ms of the final sync)."""
    import ctypes
    from evora_b200._native import lib
    p = kh_params(ev)
    sh = ev.shapes(p)
    w, evo, s = np.zeros(sh["w"]), np.zeros(sh["evo"]), np.zeros(sh["s"])
    qh = q.copy()
    di = ev.DropIn(p)
    di.set_resident(mode)
    # the C ABI called as a Fortran main program calls it: the arrays' base
    # addresses once, the scalars by reference
    L = lib()
    pw, pq, pevo, ps = (ctypes.c_void_p(a.ctypes.data) for a in (w, qh, evo, s))
    dt, t = ctypes.c_double(0.0), ctypes.c_double(p.tstart)
    go, dump, k = ctypes.c_int32(1), ctypes.c_int32(0), ctypes.c_int32(1)

    def step():
        rc = L.evora_primitive(pw, pq) | L.evora_bound(pw)
        dt.value = 1e99
        rc |= L.evora_hydrostep(pw, ctypes.byref(dt))
        rc |= L.evora_updatetime(ctypes.byref(go), ctypes.byref(dump), ctypes.byref(k), ctypes.byref(t),
                                 ctypes.byref(dt))
        rc |= L.evora_compevo(pw, pevo, ps, dt.value)
        rc |= L.evora_sweep(pw, pq, pevo, ps, dt.value)
        if rc:
            raise RuntimeError(f"drop-in step failed: status {rc}")

    try:
        for _ in range(warmup):
            step()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        t1 = time.perf_counter()
        di.sync(qh)
        t2 = time.perf_counter()
    finally:
        di.set_resident(0)
    return 1e3 * (t1 - t0) / steps, 1e3 * (t2 - t1)


def oracle_errors(q0, steps, results):
    """Relative L1 per field of GPU results against the oracle (the CPU
    restatement of the reference, all host threads) after the same steps
    from the same initial state: {name: [rho, mx, my, mz, E]}."""
    from oracle.oracle import Oracle, make_params
    o = Oracle(make_params(nx=NX, ny=NY, nz=NZ, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6))
    q = q0.copy()
    r = o.run(q, steps)
    if r["status"] or r["steps"] != steps:
        return {"error": f"oracle status {r['status']} after {r['steps']} steps"}
    out = {}
    for name, qg in results.items():
        num = np.abs(qg[..., :5] - q[..., :5]).reshape(-1, 5).sum(0)
        den = np.abs(q[..., :5]).reshape(-1, 5).sum(0)
        out[name] = [float(x) for x in np.where(den > 0, num / np.where(den > 0, den, 1.0), num)]
    return out


def reference_serial(budget_s=8.0):
    """The reference's own hydro path, translated mechanically from its
    Fortran sources (oracle/_ref), on one host thread: the analogue of one
    reference MPI rank, on a z-slab of the workload."""
    try:
        from oracle.ref_oracle import RefOracle, LIB_PATH
        if not os.path.exists(LIB_PATH):
            return None
        o = RefOracle(nx=NX, ny=NY, nz=2, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6)
        q = o.zeros_q()
        q[...] = _kh_slab(2)
        t0 = time.perf_counter()
        o.run(q, 1)
        per_cell = (time.perf_counter() - t0) / (NX * NY * 2)
        nz_s = int(max(2, min(NZ, budget_s / max(per_cell, 1e-12) / (NX * NY))))
        o = RefOracle(nx=NX, ny=NY, nz=nz_s, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6)
        q = o.zeros_q()
        q[...] = _kh_slab(nz_s)
        t0 = time.perf_counter()
        r = o.run(q, 1)
        el = time.perf_counter() - t0
        return {"value": NX * NY * nz_s * max(1, r["steps"]) / el, "unit": METRIC, "cores": 1,
                "kind": "reference",
                "sample": f"1 step of a {NX}x{NY}x{nz_s} periodic slab of the workload, FP64, the reference's "
                          f"Fortran hydro path translated to C (oracle/_ref), one thread, {el:.1f} s"}
    except Exception as e:  # the serial figure is an extra; the line does not depend on it
        return {"error": str(e)}


def _kh_slab(nz_s):
    """The KH initial state of a slab of nz_s planes (the IC is z-invariant)."""
    import evora_b200 as ev
    p = ev.default_params(nx=NX, ny=NY, nz=nz_s, g=GAMMA, cfl=CFL, boundtype=2)
    return ev.ic.kh3d(p, seed=42, amp=0.01)


def cpu_baseline(steps_budget_s=20.0, threads=None):
    """The oracle (C restatement, FP64) on all host threads, on a z-slab of
    the workload (256 x 256 x nz_s, periodic; the KH IC is z-invariant, so
    the per-cell work equals the full grid's)."""
    from oracle.oracle import Oracle, make_params
    o = Oracle(make_params(nx=NX, ny=NY, nz=8, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6))
    if threads:
        o.set_threads(threads)
    cores = o.max_threads()
    q = o.ic_kh3d(42, 0.01)
    t0 = time.perf_counter()
    o.run(q, 1)
    per_cell = (time.perf_counter() - t0) / q[..., 0].size
    nz_s = int(max(8, min(NZ, steps_budget_s / 3.0 / max(per_cell, 1e-12) / (NX * NY))))
    o = Oracle(make_params(nx=NX, ny=NY, nz=nz_s, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6))
    q = o.ic_kh3d(42, 0.01)
    o.run(q, 1)   # warm
    t0 = time.perf_counter()
    r = o.run(q, 2)
    el = time.perf_counter() - t0
    cells = NX * NY * nz_s * r["steps"]
    return {"value": cells / el, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"2 steps of a {NX}x{NY}x{nz_s} periodic slab of the workload, FP64, "
                      f"OpenMP over pencils ({cores} threads), {el:.1f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import Oracle, make_params
    probe = Oracle(make_params(nx=NX, ny=NY, nz=4, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6))
    cores = probe.max_threads()
    q = probe.ic_kh3d(42, 0.01)
    t0 = time.perf_counter()
    probe.run(q, 1)
    per_cell = (time.perf_counter() - t0) / q[..., 0].size
    budget = 150.0 / max(1, args.steps + args.warmup)       # seconds per step
    nz_s = int(max(4, min(NZ, budget / max(per_cell, 1e-12) / (NX * NY))))
    o = Oracle(make_params(nx=NX, ny=NY, nz=nz_s, g=GAMMA, cfl=CFL, boundtype=2, tend=1e6))
    q = o.ic_kh3d(42, 0.01)
    o.run(q, args.warmup)
    t0 = time.perf_counter()
    r = o.run(q, args.steps)
    el = time.perf_counter() - t0
    value = NX * NY * nz_s * r["steps"] / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / max(1, r["steps"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sample_nz": nz_s},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} steps of a {NX}x{NY}x{nz_s} periodic slab of the "
                                   f"workload (z-invariant IC), FP64, OpenMP over pencils"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def front_position(rho, i):
    """Sub-cell position of the density front around the jump between cells
    i and i+1: where the profile crosses the mean of the densities three
    cells either side (linear between cells)."""
    n = len(rho)
    a, b = rho[max(i - 3, 0)], rho[min(i + 4, n - 1)]
    level = 0.5 * (a + b)
    for k in range(max(i - 3, 0), min(i + 4, n - 1)):
        if (rho[k] - level) * (rho[k + 1] - level) <= 0 and rho[k + 1] != rho[k]:
            return k + (level - rho[k]) / (rho[k + 1] - rho[k])
    return float(i) + 0.5


def front_shift(rho, rho_ref, lo=0):
    """Cells between the largest density jump of rho_ref (beyond index lo)
    and the same front in rho."""
    i = lo + int(np.argmax(np.abs(np.diff(rho_ref[lo:]))))
    return abs(front_position(rho, i) - front_position(rho_ref, i))


def run_sod(args):
    """The 1D Sod shock tube of the reference's shock-tube test (1024 cells
    on [0, 1], gamma 1.4, (1, 0, 1) | (0.125, 0, 0.1) at x = 0.5, outflow,
    minmod, HLLC, CFL 0.8, to t = 0.2): each form against the oracle, L1
    density and the shock position in cells; device time of the whole run."""
    import torch
    import evora_b200 as ev
    from oracle.oracle import Oracle, make_params
    dist_setup(args.gpus)
    kw = dict(nx=1024, ny=1, nz=1, g=1.4, cfl=0.8, boundtype=1, solver=2, limiter=1, tend=0.2)
    p = ev.default_params(**kw)
    q0 = ev.ic.shocktube(p)
    o = Oracle(make_params(**kw))
    qo = q0.copy()
    r = o.run(qo, 1 << 30)
    rho_o = qo[0, 0, :, 0]
    forms = {}
    for name, prec, flags in (("fp64_strict", ev.FP64, ev.STRICT), ("fp64", ev.FP64, 0), ("fp32", ev.FP32, 0)):
        stream = torch.cuda.Stream()
        with ev.Grid(p, prec, flags) as g:
            g.set_stream(stream)
            for _ in range(max(3, args.warmup)):   # whole runs from the IC
                g.set_q(q0)
                g.run()
            g.set_q(q0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t = g.run()
            e1.record(stream)
            torch.cuda.synchronize()
            rho = g.get_q()[0, 0, :, 0]
        forms[name] = {"steps": t["k"], "t": t["t"], "ms_run": e0.elapsed_time(e1),
                       "l1_density_vs_oracle": float(np.abs(rho - rho_o).sum() / np.abs(rho_o).sum()),
                       "shock_shift_cells": float(front_shift(rho, rho_o, lo=int(0.75 * kw["nx"]))),
                       "bitwise_rho_m_e": bool(np.array_equal(rho, rho_o))}
    v = forms["fp32"]
    line = {"metric": METRIC, "value": kw["nx"] * v["steps"] / (v["ms_run"] * 1e-3), "unit": METRIC, "n_gpus": 1,
            "steps": v["steps"], "warmup": max(3, args.warmup), "ms_per_step": v["ms_run"] / v["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "1D Sod shock tube, 1024 cells, gamma 1.4, outflow, minmod, HLLC, CFL 0.8, "
                                   "t = 0.2 (one grid; a whole run is timed)"},
            "oracle": {"steps": r["steps"], "t": r["t"]}, "forms": forms}
    print(json.dumps(line), flush=True)
    return 0


def run_tubes(args):
    """Batched Riemann problems: ntubes independent 1D tubes, lengths uniform
    in [128, 4096], random left/right states (rho, p log-uniform, v uniform,
    interface in [0.3, 0.7]), gamma 5/3, CFL 0.8, every tube advanced to
    t = 0.1 in one persistent launch; HLLC and HLL, FP32 (and FP64 for the
    error).  One timed launch = the whole job; warm-up launches on the same
    data are discarded."""
    import torch
    import evora_b200 as ev
    from evora_b200 import sharding
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    lengths_all, q_all = ev.ic.random_tubes(args.ntubes, seed=7, nmin=128, nmax=4096)
    # N > 1: whole tubes per rank, balanced by estimated work; no exchange
    shards = sharding.shard_by_work(sharding.tube_work(lengths_all, q_all), world)
    lengths, q = sharding.pack(lengths_all, q_all, shards[rank])
    cells = sum(lengths_all)
    res = {}
    for solver in (2, 1):
        p = ev.default_params(nx=max(lengths), ny=1, nz=1, g=5.0 / 3.0, cfl=0.8, boundtype=1,
                              solver=solver, tend=0.1)
        out = {}
        for prec, name in ((ev.FP32, "f32"), (ev.FP64, "f64")):
            stream = torch.cuda.Stream()
            with ev.Batch(p, lengths, prec) as b:
                b.set_stream(stream)
                b.set_q(q)
                tune = b.autotune(steps=20)
                for _ in range(max(3, args.warmup)):   # warm-up (graph capture, caches)
                    b.set_q(q)
                    b.run()
                ms_runs, work = [], 0
                for _ in range(max(1, args.steps)):
                    b.set_q(q)                # every timed run starts from the initial tubes
                    cu0 = b.cell_updates()
                    s0 = torch.cuda.Event(enable_timing=True)
                    s1 = torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    s0.record(stream)
                    b.run(sync=False)
                    s1.record(stream)
                    torch.cuda.synchronize()
                    ms_runs.append(s0.elapsed_time(s1))
                    work += b.cell_updates() - cu0
                runs = len(ms_runs)
                ms = sharding.max_over_ranks(float(np.mean(ms_runs)), dev)
                work = sharding.sum_over_ranks(work / runs, dev)
                infos = [b.info(i) for i in range(len(lengths))]
                qq = b.get_q()
            failed = int(sharding.sum_over_ranks(sum(1 for i in infos if i["status"] == 2), dev))
            steps = [i["k"] for i in infos]
            out[name] = {"value": work / (ms * 1e-3), "ms": ms, "cell_updates": work, "failed_tubes": failed,
                         "steps_min": min(steps), "steps_max": max(steps), "autotune": tune, "q": qq,
                         "ok": [i["status"] == 1 for i in infos]}
        offs = np.concatenate([[0], np.cumsum(lengths)])
        l1 = []
        for i in range(len(lengths)):
            if out["f32"]["ok"][i] and out["f64"]["ok"][i]:
                a, b64 = out["f32"]["q"][offs[i]:offs[i + 1], 0], out["f64"]["q"][offs[i]:offs[i + 1], 0]
                l1.append(np.abs(a - b64).sum() / np.abs(b64).sum())
        vs_oracle = None
        if world == 1 and not args.no_oracle_check:
            # every tube against the oracle (spawned pool over tubes): L1
            # density and the shift of its largest density jump, in cells
            from oracle.oracle import run_tubes as oracle_tubes
            ref = oracle_tubes(dict(g=5.0 / 3.0, cfl=0.8, boundtype=1, solver=solver, tend=0.1), lengths, q)
            vs_oracle = {}
            for name in ("f32", "f64"):
                e, sh, same_steps = [], [], 0
                for i, (qo, ri) in enumerate(ref):
                    if ri["status"] or not out[name]["ok"][i]:
                        continue
                    a = out[name]["q"][offs[i]:offs[i + 1], 0]
                    e.append(np.abs(a - qo[:, 0]).sum() / np.abs(qo[:, 0]).sum())
                    sh.append(front_shift(a, qo[:, 0]))
                vs_oracle[name] = {"tubes": len(e), "l1_density_median": float(np.median(e)),
                                   "l1_density_max": float(np.max(e)),
                                   "front_shift_cells_median": float(np.median(sh)),
                                   "front_shift_cells_max": float(np.max(sh)),
                                   "oracle_failed_tubes": sum(1 for _, ri in ref if ri["status"])}
        for v in out.values():
            v.pop("q")
            v.pop("ok")
        res["hllc" if solver == 2 else "hll"] = dict(
            out, l1_density_f32_vs_f64_median=float(np.median(l1)) if l1 else None,
            l1_density_f32_vs_f64_max=sharding.max_over_ranks(float(np.max(l1)) if l1 else 0.0, dev),
            vs_oracle=vs_oracle)
    peak, peak_kind = measured_peaks()
    v = res["hllc"]["f32"]
    if rank != 0:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
        return 0
    line = {"metric": METRIC, "value": v["value"], "unit": METRIC, "n_gpus": world, "steps": max(1, args.steps),
            "warmup": max(3, args.warmup),
            "ms_per_step": v["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.ntubes} batched 1D Riemann tubes, 128-4096 cells, to t=0.1, "
                                   "gamma 5/3, CFL 0.8, HLLC (HLL below)", "cells": cells,
                       "step": "one persistent launch advancing every tube to t=0.1 (state reset between "
                               "timed launches)",
                       "l2": "inputs larger than L2 (175 MB FP32 state)"},
            "roofline": {"bound": "hbm", "achieved": cells * 40 / (v["ms"] * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": cells * 40 / (v["ms"] * 1e-3) / 1e9 / peak, "traffic": None,
                         "peak_kind": peak_kind,
                         "note": "each tube crosses HBM once per launch; the kernel is compute bound"},
            "tubes": res}
    if world > 1:
        line["scaling"] = "strong"
        line["config"]["parallelism"] = f"tubes sharded by estimated work over {world} ranks, no exchange"
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


# Algorithmic bytes per cell of the gravity substep: mean of rho (read rho),
# source (read rho, write phi FP64), D2Z (read phi, write the half
# spectrum), Green's factor (read + write it), Z2D (read it, write phi),
# integration (read rho, m, E and phi, write m and E).
GRAV_BYTES = {"f32": 4 + 12 + 16 + 16 + 16 + (20 + 8 + 16), "f64": 8 + 16 + 16 + 16 + 16 + (40 + 8 + 32)}
# conduction substep: primitives and T (read 5 fields, write T FP64), update
# (read T, rho, E, write E)
COND_BYTES = {"f32": (20 + 8) + (8 + 4 + 4 + 4), "f64": (40 + 8) + (8 + 8 + 8 + 8)}
# KH box edge for the conduction workload: kappa_eff = 1/(g-1) is explicit,
# and a 640-unit box keeps its diffusion number near 0.1 at the hydro step
COND_BOX = 640.0
# comoving substeps: gravity from the comoving source (no mean-density pass)
# and the expansion terms (read rho, m, E, write E)
COMOV_BYTES = {"f32": GRAV_BYTES["f32"] - 4 + (20 + 4), "f64": GRAV_BYTES["f64"] - 8 + (40 + 8)}
# a comoving run from z = 99 (omega0 = 1): the expansion's step limit
# (cosmostep) stays far above the hydro step, so both grids take the same dt
COMOVING = dict(supercomoving=1, omega0=1.0, lambda0=0.0, zstart=99.0, zend=0.0, gravity=1)


def run_physics(args, kind):
    """The KH workload with more physics after every hydro step: gravity
    (gravitation.f90, non-comoving: FFT Poisson solve with cuFFT D2Z/Z2D in
    FP64 and the force update), thermal conduction (conduction.f90
    simplekappa, with thermalstep in the CFL kernel), or comoving coordinates
    (the expansion factor integrated in the control kernel, gravity from the
    comoving source and the expansion terms, main.f90:124-178).  Reports
    cell-updates/s of whole steps and the substeps' time (grid with them
    minus grid without, same box) against their algorithmic bytes."""
    import torch
    import evora_b200 as ev
    world, rank, local = dist_setup(args.gpus)
    stream = torch.cuda.Stream()
    q = ev.ic.kh3d(kh_params(ev), seed=42, amp=0.01)
    n = NX * NY * NZ
    peak, peak_kind = measured_peaks()
    nbytes = {"gravity": GRAV_BYTES, "conduction": COND_BYTES, "comoving": COMOV_BYTES}[kind]
    box = COND_BOX if kind == "conduction" else 1.0
    extra = {"gravity": {"gravity": 1}, "conduction": {"conduction": 1}, "comoving": COMOVING}[kind]
    out = {}
    barrier(world)
    with ClockSampler(local) as clk:
        clk.wait_first_sample()
        for prec, name in ((ev.FP32, "f32"), (ev.FP64, "f64")):
            ms_h, kt_h, g = time_grid(ev, torch, q, prec, args.steps, args.warmup, stream, box=box)
            g.close()
            ms_x, kt_x, g = time_grid(ev, torch, q, prec, args.steps, args.warmup, stream, box=box, **extra)
            g.close()
            ms_h, ms_x = max_over_ranks(world, ms_h), max_over_ranks(world, ms_x)
            sub_ms = (ms_x - ms_h) / args.steps
            achieved = n * nbytes[name] / (sub_ms * 1e-3) / 1e9 if sub_ms > 0 else None
            out[name] = {"value": world * n * args.steps / (ms_x * 1e-3), "ms_per_step": ms_x / args.steps,
                         "hydro_ms_per_step": ms_h / args.steps, f"{kind}_ms_per_step": sub_ms,
                         f"{kind}_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                              "frac": achieved / peak if achieved else None,
                                              "algorithmic_bytes_per_cell": nbytes[name],
                                              "peak_kind": peak_kind},
                         "gpu_launches": kt_x["launches"]}
    if rank == 0:
        v = out["f32"]
        what = {"gravity": "self-gravity after every step (FFT Poisson solve, FP64)",
                "conduction": f"thermal conduction after every step (simplekappa, box {COND_BOX:g})",
                "comoving": "comoving coordinates from z = 99 (omega0 = 1): expansion factor, comoving "
                            "gravity and expansion terms with every step"}[kind]
        line = {"metric": METRIC, "value": v["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": v["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD + ", " + what, "cells": n, "l2": "inputs larger than L2"},
                "roofline": v[f"{kind}_roofline"], kind: out, "gpu_launches": v["gpu_launches"],
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cosmo_params(ev):
    """The comoving box: 256^3 periodic, gamma 5/3, HLLC/minmod, CFL 0.5,
    omega0 0.3, lambda0 0.7, H0 70, 20 Mpc/h, fb 0.17, from z = 50, with
    comoving gravity and the expansion terms; c_cosmo 0.01 (a grows by at
    most 1% per step, so 200 steps stay far from z = 0); dual energy with
    de_thresh 1e-3 (the gas is cold: T = 100 K against Zel'dovich flows of
    Mach ~50, so E - kin is kept through the entropy where it is below a
    thousandth of E, comp.f90:45-85)."""
    return ev.default_params(nx=NX, ny=NY, nz=NZ, g=GAMMA, cfl=CFL, boundtype=2, solver=2, limiter=1,
                             supercomoving=1, gravity=1, omega0=0.3, lambda0=0.7, hubble0=70.0, box=20.0,
                             zstart=50.0, zend=0.0, fb=0.17, c_cosmo=0.01, dualenergy=1, de_thresh=1e-3,
                             chemistry=int(CHEMISTRY), cooling=int(CHEMISTRY))


def run_cosmo(args):
    """The comoving cosmological box: Zel'dovich IC from a
    seeded power law P(k) ~ k^-2 at z = 50 (ic/cosmo.f90's construction,
    density rms 0.05), T = 100 K, 200 steps of hydro + comoving gravity
    (cuFFT) + expansion terms and, unless --no-chemistry, the six CIE species
    with FP64 cooling, FP32 and FP64.  Reports cell-updates/s, the
    fused update's share and roofline, the substeps' time, the redshift
    reached and the FP32 density error against FP64."""
    import torch
    import evora_b200 as ev
    world, rank, local = dist_setup(args.gpus)
    stream = torch.cuda.Stream()
    steps = args.steps if args.steps != 100 else 200
    p = cosmo_params(ev)
    q = ev.ic.cosmo_zeldovich(p, seed=5, slope=-2.0, sigma=0.05, temp_k=100.0)
    n = NX * NY * NZ
    peak, peak_kind = measured_peaks()
    out, rho = {}, {}
    barrier(world)
    with ClockSampler(local) as clk:
        clk.wait_first_sample()
        for prec, name in ((ev.FP32, "f32"), (ev.FP64, "f64")):
            g = ev.Grid(p, prec)
            g.set_stream(stream)
            g.set_q(q)
            g.step(args.warmup, sync=True)
            tune = pick_tile(g, prec)
            torch.cuda.synchronize()
            g.set_timing(True)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            g.step(steps, sync=False)
            end.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(world, start.elapsed_time(end))
            kt, st = g.timing(), g.status()
            if st:
                raise RuntimeError(f"cosmological box stopped with status {st}")
            s, _ = g.cosmo()
            rho[name] = g.get_q()[..., 0].copy()
            # the fused update of the 6-field (dual-energy) state: 6 fields
            # read and written once
            upd_ms = kt["fused_ms"] / max(kt["steps"], 1)
            phys_ms = kt["physics_ms"] / max(kt["steps"], 1)
            achieved = n * (48 if name == "f32" else 96) / (upd_ms * 1e-3) / 1e9
            out[name] = {"value": world * n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                         "update_kernel_ms": upd_ms, "gravity_expansion_ms": phys_ms,
                         "cfl_ms": kt["cfl_ms"] / max(kt["steps"], 1),
                         "redshift_reached": s["redshift"], "steps_timed": g.time()["k"] - args.warmup,
                         "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                      "frac": achieved / peak, "peak_kind": peak_kind},
                         "gpu_launches": kt["launches"],
                         "autotune": {"chosen": tune[0], "ms_per_tile": tune[1]}}
            g.close()
    if rank == 0:
        v = out["f32"]
        l1 = float(np.abs(rho["f32"] - rho["f64"]).sum() / np.abs(rho["f64"]).sum())
        line = {"metric": METRIC, "value": v["value"], "unit": METRIC, "n_gpus": world, "steps": steps,
                "warmup": args.warmup, "ms_per_step": v["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"3D comoving cosmological box {NX}^3 periodic, gamma=5/3, Zel'dovich IC from "
                                       "a seeded power law P(k)~k^-2 at z=50 (density rms 0.05), fb=0.17, T=100 K, "
                                       "omega0=0.3, lambda0=0.7, H0=70, 20 Mpc/h; cuFFT comoving gravity and "
                                       "expansion terms; " + ("six species in CIE with FP64 per-cell cooling "
                                                              "(neutral start)" if CHEMISTRY else
                                                              "without chemistry (--no-chemistry)"),
                           "cells": n, "l2": "inputs larger than L2"},
                "roofline": v["roofline"], "cosmo": out, "l1_density_fp32_vs_fp64": l1,
                "gpu_launches": v["gpu_launches"], "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serving_requests(ev, n, seed=11):
    """The serving mix: 60% 1D tubes of 128-8192 cells (random Riemann states
    as in the batched workload, to t=0.05), 30% 2D Kelvin-Helmholtz
    64^2-1024^2 (ic/kevinhelmholtz.f90 IC, to t=0.02), 10% 3D Kelvin-Helmholtz
    32^3-128^3 (seeded IC, to t=0.02).  The 2D/3D edge lengths are drawn on a
    16-cell grid so that one initial state per size is kept (host memory
    stays bounded for thousands of requests)."""
    rng = np.random.default_rng(seed)
    cache = {}
    reqs = []
    for _ in range(n):
        u = rng.random()
        if u < 0.6:
            m = int(rng.integers(128, 8193))
            _, q = ev.ic.random_tubes(1, seed=int(rng.integers(1 << 30)), nmin=m, nmax=m)
            reqs.append(("1d", q.reshape(1, 1, m, 6), 0.05))
        elif u < 0.9:
            m = 16 * int(rng.integers(4, 65))
            if ("2d", m) not in cache:
                cache[("2d", m)] = ev.ic.kh2d(ev.default_params(nx=m, ny=m, nz=1, g=5.0 / 3.0))
            reqs.append(("2d", cache[("2d", m)], 0.02))
        else:
            m = 16 * int(rng.integers(2, 9))
            if ("3d", m) not in cache:
                cache[("3d", m)] = ev.ic.kh3d(ev.default_params(nx=m, ny=m, nz=m, g=5.0 / 3.0), seed=m)
            reqs.append(("3d", cache[("3d", m)], 0.02))
    return reqs


def serve(server, reqs, arrivals, keep=(), borrowed=True):
    """Submits requests at their arrival times (host clock) to the server and
    ticks it until all are done.  borrowed: each request's state is read, and
    its result written into an array of its own, by the server's copy
    threads while the device works (Server.submit_borrowed); else the state
    is copied at submit and results are read into reused buffers, one per
    shape.  The results of the requests in `keep` are kept.  Returns
    latencies by kind, the wall time, cell-updates, rounds, mean round time,
    round phases and the kept results."""
    lat = {"1d": [], "2d": [], "3d": []}
    kept, bufs = {}, {}
    cu0 = server.stats()["cell_updates"]
    ph0 = server.profile()
    t0 = time.perf_counter()
    nxt, done, ticks, tick_s, submit_s, deliver_s = 0, 0, 0, 0.0, 0.0, 0.0
    slow = []   # (seconds, cells) per submit call
    ids = {}
    while done < len(reqs):
        now = time.perf_counter() - t0
        ts = time.perf_counter()
        while nxt < len(reqs) and arrivals[nxt] <= now:
            kind, q, tend = reqs[nxt]
            bt = 1 if kind == "1d" else 2
            t1 = time.perf_counter()
            if borrowed:
                ids[server.submit_borrowed(q, tend, boundtype=bt, out=np.empty(q.shape))] = nxt
            else:
                ids[server.submit(q, tend, boundtype=bt)] = nxt
            slow.append((time.perf_counter() - t1, q.size // 6))
            nxt += 1
        tk = time.perf_counter()
        submit_s += tk - ts
        a, p = server.tick()
        td = time.perf_counter()
        tick_s += td - tk
        ticks += 1
        for rid in server.completed():
            i = ids.pop(rid)
            shape = reqs[i][1].shape
            if borrowed:
                out = None
            elif i in keep:
                out = np.empty(shape)
            else:
                out = bufs.setdefault(shape, np.empty(shape))
            r = server.result(rid, out=out)
            lat[reqs[i][0]].append(r[1])
            if i in keep:
                kept[i] = (r[0], r[3])
            done += 1
        deliver_s += time.perf_counter() - td
        if a == 0 and p == 0 and nxt < len(reqs):
            time.sleep(max(0.0, min(0.01, arrivals[nxt] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    ph = server.profile()
    phases = {k: ph[k] - ph0[k] for k in ph}
    phases["submit"] = submit_s      # submit calls (with borrowed=False: the copy into the page-locked pool)
    phases["deliver"] = deliver_s    # completed() and result() (with borrowed=False: the copy out of it)
    phases["submit_slowest_ms_cells"] = [[1e3 * t, c] for t, c in sorted(slow, reverse=True)[:4]]
    cu = server.stats()["cell_updates"] - cu0
    return lat, wall, cu, ticks, 1e3 * tick_s / max(1, ticks), phases, kept


def run_serving(args):
    """Serving mix (serving_requests) with Poisson arrivals, FP32, admitted
    under a 150 GB HBM budget with the state kept resident; p50/p99 time to
    solution (submit to read-back) and the aggregate cell-updates/s.  With
    --sustained: first the capacity (all requests of a burst of --nrequests
    at once, requests per second completed), then >= 2000 requests arriving
    at 70% of that rate, whose latencies are the ones to quote.  A few small
    requests are rerun alone in FP64 as spot checks of the FP32 results."""
    import evora_b200 as ev
    from evora_b200 import sharding
    from evora_b200.serving import Server
    world, rank, local = dist_setup(args.gpus)
    pct = lambda a, f: float(np.percentile(a, f)) if a else None  # noqa: E731

    def serve_sharded(reqs, arrivals, keep=()):
        """serve() over the ranks: each request to the least-loaded rank in
        arrival order (sharding.assign_online), all ranks starting together;
        latencies, cell-updates and phases gathered on rank 0, the wall
        time the max over ranks."""
        owner = sharding.assign_online([sharding.request_work(r[1].shape, r[2]) for r in reqs], world)
        mine = [i for i in range(len(reqs)) if owner[i] == rank]
        barrier(world)
        lat, wall, cu, ticks, mround, phases, kept = serve(server, [reqs[i] for i in mine],
                                                           np.asarray(arrivals)[mine],
                                                           keep={k for k, i in enumerate(mine) if i in keep},
                                                           borrowed=not args.copy_at_submit)
        kept = {mine[k]: v for k, v in kept.items()}
        parts = sharding.gather_objects((lat, wall, cu, ticks, mround, phases), rank, world)
        if rank != 0:
            return None
        lat = {k: sum((pt[0][k] for pt in parts), []) for k in ("1d", "2d", "3d")}
        wall = max(pt[1] for pt in parts)
        cu = sum(pt[2] for pt in parts)
        ticks = max(pt[3] for pt in parts)
        mround = max(pt[4] for pt in parts)
        phases = {k: max(pt[5][k] for pt in parts) for k in parts[0][5] if k != "submit_slowest_ms_cells"}
        phases["submit_slowest_ms_cells"] = sorted((x for pt in parts for x in pt[5]["submit_slowest_ms_cells"]),
                                                   reverse=True)[:4]
        return lat, wall, cu, ticks, mround, phases, kept

    def summary(lat):
        allat = sorted(lat["1d"] + lat["2d"] + lat["3d"])
        return {"p50": pct(allat, 50), "p99": pct(allat, 99),
                "by_kind": {k: {"n": len(v), "p50": pct(v, 50), "p99": pct(v, 99)} for k, v in lat.items()}}

    out = {}
    rate = args.rate
    nreq = args.nrequests
    # one server for the whole run (as a service keeps it); a first pass of
    # the mix warms it (graphs, page-locked buffers) and is not reported
    server = Server(ev.default_params(g=5.0 / 3.0, cfl=0.5, boundtype=1, tend=1.0), ev.FP32, 0,
                    hbm_budget_bytes=150e9, steps_per_tick=args.tick_steps, max_tube_cells=8192, max_tubes=4096)
    # twice as many requests as the burst below, all at once, so that the
    # page-locked pool holds the buffers a burst of the mix keeps at once
    # (pinning memory is a service's one-time start-up cost: 54-111 ms per
    # 128^3 state measured in a submit call)
    warm = serving_requests(ev, 2 * args.nrequests, seed=10)
    serve(server, warm, np.zeros(len(warm)), borrowed=not args.copy_at_submit)
    if args.sustained:
        burst = serving_requests(ev, args.nrequests, seed=11)
        res = serve_sharded(burst, np.zeros(len(burst)))
        capacity = 0.0
        if rank == 0:
            lat, wall, cu, ticks, mround, phases, _ = res
            capacity = len(burst) / wall
            out["capacity"] = {"requests": len(burst), "requests_per_s": capacity, "cell_updates_per_s": cu / wall,
                               "wall_s": wall, "round_phases_s": phases, "latency_s": summary(lat)}
        rate = 0.7 * max_over_ranks(world, capacity)   # rank 0's, on every rank
        nreq = max(2000, args.nrequests)
    rng = np.random.default_rng(12)
    reqs = serving_requests(ev, nreq, seed=13 if args.sustained else 11)
    small = [i for i, r in enumerate(reqs) if r[1].size <= 6 * 300_000][:8]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    res = serve_sharded(reqs, arrivals, keep=set(small))
    server.close()
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return 0
    lat, wall, cu, ticks, mround, phases, results = res
    # FP64 spot checks of small FP32 results (alone, same server options)
    checks = []
    for i in small:
        kind, q, tend = reqs[i]
        if len(checks) >= 4:
            break
        if i not in results:   # served by another rank
            continue
        q32, err = results[i]
        if err:
            continue
        bt = 1 if kind == "1d" else 2
        with Server(ev.default_params(g=5.0 / 3.0, cfl=0.5, boundtype=1, tend=1.0), ev.FP64,
                    0, hbm_budget_bytes=10e9, steps_per_tick=256, max_tube_cells=8192, max_tubes=4) as s64:
            rid = s64.submit(q, tend, boundtype=bt)
            while s64.tick() != (0, 0):
                pass
            q64 = s64.result(rid)[0]
        checks.append({"kind": kind, "cells": int(q.size // 6),
                       "l1_density_f32_vs_f64": float(np.abs(q32[..., 0] - q64[..., 0]).sum()
                                                      / np.abs(q64[..., 0]).sum())})
    line = {"metric": METRIC, "value": cu / wall, "unit": METRIC, "n_gpus": world, "steps": len(reqs), "warmup": 0,
            "ms_per_step": 1e3 * wall / len(reqs), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "serving mix: 60% 1D tubes 128-8192, 30% 2D KH 64^2-1024^2, 10% 3D KH "
                                   "32^3-128^3, Poisson arrivals", "rate_per_s": rate,
                       "requests": len(reqs), "tick_steps": args.tick_steps, "hbm_budget_gb": 150,
                       "arrivals": "70% of the measured capacity" if args.sustained else "--rate",
                       "host_copies": ("at submit and delivery on the driving thread" if args.copy_at_submit else
                                       "borrowed arrays, copied by the server's threads while the device works"),
                       "parallelism": (f"requests dispatched to the least-loaded of {world} ranks on arrival, "
                                       "no exchange") if world > 1 else "single GPU"},
            "latency_s": summary(lat),
            "wall_s": wall, "cell_updates": cu, "rounds": ticks, "mean_round_ms": mround,
            "round_phases_s": phases, "spot_checks_fp64": checks, **out}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the full-size comparison of both forms with the CPU oracle")
    ap.add_argument("--size", type=int, default=256,
                    help="cells per axis (256 = the benchmark; smaller sizes for ncu captures)")
    ap.add_argument("--forms", default="f32,f64", help="f32,f64 (default) or f32 alone")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tile shape")
    ap.add_argument("--tiles", default=None,
                    help="F32,F64: pin the fused kernel's tile shapes (indices of the tile table) instead of autotune")
    ap.add_argument("--workload", default="kh3d",
                    choices=["kh3d", "sod", "tubes", "serving", "gravity", "conduction", "comoving", "cosmo"],
                    help="kh3d: the benchmark (256^3 KH); tubes: 4096 batched Riemann tubes; serving: request "
                         "mix; gravity / conduction / comoving: the KH benchmark with those substeps after every "
                         "step; cosmo: the comoving cosmological box (Zel'dovich IC, 200 steps)")
    ap.add_argument("--ntubes", type=int, default=4096)
    ap.add_argument("--rate", type=float, default=200.0, help="serving: arrivals per second")
    ap.add_argument("--nrequests", type=int, default=400)
    ap.add_argument("--tick-steps", type=int, default=32)
    ap.add_argument("--sustained", action="store_true",
                    help="serving: measure the capacity with a burst, then latency at 70%% of it")
    ap.add_argument("--copy-at-submit", action="store_true",
                    help="serving: copy each request's state at submit and its result at delivery on the "
                         "driving thread (Server.submit) instead of the borrowed arrays of Server.submit_borrowed")
    ap.add_argument("--no-chemistry", action="store_true", help="cosmo: without the CIE chemistry and cooling")
    args = ap.parse_args()
    global NX, NY, NZ, AUTOTUNE, CHEMISTRY, WORKLOAD, TILES
    NX = NY = NZ = args.size
    WORKLOAD = WORKLOAD.replace("256^3", f"{NX}^3")
    AUTOTUNE = not args.no_autotune
    TILES = tuple(int(t) for t in args.tiles.split(",")) if args.tiles else None
    CHEMISTRY = not args.no_chemistry
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "tubes":
        return run_tubes(args)
    if args.workload == "sod":
        return run_sod(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload in ("gravity", "conduction", "comoving"):
        return run_physics(args, args.workload)
    if args.workload == "cosmo":
        return run_cosmo(args)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import evora_b200 as ev

    world, rank, local = dist_setup(args.gpus)
    stream = torch.cuda.Stream()
    p = kh_params(ev)
    q = ev.ic.kh3d(p, seed=42, amp=0.01)
    n = NX * NY * NZ

    forms = args.forms.split(",")
    barrier(world)
    with ClockSampler(local) as clk:
        clk.wait_first_sample()
        ms32, kt32, g32 = time_grid(ev, torch, q, ev.FP32, args.steps, args.warmup, stream)
        ms32 = max_over_ranks(world, ms32)
        barrier(world)
        if "f64" in forms:
            ms64, kt64, g64 = time_grid(ev, torch, q, ev.FP64, args.steps, args.warmup, stream)
            ms64 = max_over_ranks(world, ms64)
    clocks = clk.summary()
    if "f64" not in forms:
        g32.close()
        print(json.dumps({"metric": METRIC, "value": world * n * args.steps / (ms32 * 1e-3),
                          "unit": METRIC, "note": "profiling run (FP32 only)"}), flush=True)
        return 0
    # accuracy of the FP32 form against FP64 after the same steps
    tune32, tune64 = g32.tuning, g64.tuning
    q32_end, q64_end = g32.get_q(), g64.get_q()
    r32, r64 = q32_end[..., 0], q64_end[..., 0]
    l1 = float(np.abs(r32 - r64).sum() / np.abs(r64).sum())
    g32.close()
    g64.close()

    peak, peak_kind = measured_peaks()
    value32 = world * n * args.steps / (ms32 * 1e-3)
    value64 = world * n * args.steps / (ms64 * 1e-3)

    def roofline(kt, dtype, prof):
        avg_ms = kt["fused_ms"] / max(1, kt["steps"])
        bytes_alg = n * BYTES_PER_CELL[dtype]
        achieved = bytes_alg / (avg_ms * 1e-3) / 1e9
        traffic = profile_traffic(prof)
        kern = "k_fused_pair (fused MUSCL-Hancock update, two cells per thread)" if "pair" in prof else \
            "k_fused (fused MUSCL-Hancock update)"
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": f"profiles/{prof} (one ncu capture of this kernel on this "
                                                      "workload; not measured in this run)",
                "peak_kind": peak_kind, "kernel": kern,
                "kernel_ms": avg_ms, "cfl_kernel_ms": kt["cfl_ms"] / max(1, kt["steps"]),
                "algorithmic_bytes_per_launch": bytes_alg}

    line = {
        "metric": METRIC, "value": value32, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": n, "form": "FP32 state, FP64 pressure recovery (kin>E/2) and "
                   "CFL reduction", "l2": "inputs larger than L2 (335 MB FP32 / 671 MB FP64 state per copy)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": roofline(kt32, "f32", "fused_pair_kh256_fp32.md" if tune32[0] == ev.FP32_PAIR_TILE
                             else "fused_update_kh256_fp32.md"),
        "fp64": {"value": value64, "ms_per_step": ms64 / args.steps,
                 "roofline": roofline(kt64, "f64", "fused_update_kh256_fp64.md")},
        "fp32_over_fp64": value32 / value64,
        "autotune": {"fp32": {"chosen": tune32[0], "ms_per_tile": tune32[1]},
                     "fp64": {"chosen": tune64[0], "ms_per_tile": tune64[1]}},
        "l1_density_fp32_vs_fp64": l1,
        "gpu_launches": kt32["launches"],
        "clocks": clocks,
    }
    if not args.no_e2e and rank == 0:
        qp = torch.empty(q.shape, dtype=torch.float64, pin_memory=True).numpy()
        qp[...] = q
        outs = [torch.empty(q.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
        e2e_steps = max(4, min(args.steps, 10))
        note = (f"per step: q(6,{NX}^3) FP64 from pinned host -> set_q, 1 step, get_q -> pinned host; two grids "
                "on two streams alternate the steps so uploads overlap downloads")
        el = time_e2e(ev, torch, qp, outs, ev.FP32, e2e_steps)
        line["e2e"] = {"value": n * e2e_steps / el, "unit": METRIC, "h2d_bytes_per_step": q.nbytes,
                       "d2h_bytes_per_step": q.nbytes, "form": "FP32", "note": note}
        el64 = time_e2e(ev, torch, qp, outs, ev.FP64, e2e_steps)
        line["fp64"]["e2e"] = {"value": n * e2e_steps / el64, "unit": METRIC, "h2d_bytes_per_step": q.nbytes,
                               "d2h_bytes_per_step": q.nbytes, "form": "FP64", "note": note}
    if not args.no_e2e and rank == 0:
        # the unmodified driver's call sequence with host arrays, state resident
        line["dropin_resident"] = {}
        for mode, name, ms_grid in ((ev.RESIDENT_FP32, "fp32", ms32 / args.steps),
                                    (ev.RESIDENT_FP64, "fp64", ms64 / args.steps)):
            ms_step, ms_sync = time_dropin_resident(ev, q, mode, args.steps, args.warmup)
            line["dropin_resident"][name] = {
                "ms_per_step": ms_step, "grid_ms_per_step": ms_grid, "over_grid": ms_step / ms_grid,
                "final_sync_ms": ms_sync, "value": n / (ms_step * 1e-3), "unit": METRIC,
                "note": "host wall time of primitive, bound, hydrostep, updatetime, compevo, sweep per step "
                        "(main.f90:109-155) on host arrays in resident mode; evora_sync of q once at the end"}
    if rank == 0 and world == 1 and not args.no_oracle_check:
        # both forms against the oracle after the same steps (autotune keeps the state)
        line["l1_vs_oracle"] = {"steps": args.warmup + args.steps, "fields": ["rho", "mx", "my", "mz", "E"],
                                **oracle_errors(q, args.warmup + args.steps, {"fp32": q32_end, "fp64": q64_end})}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
        serial = reference_serial()
        if serial:
            line["cpu_baseline"]["reference_serial"] = serial
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
