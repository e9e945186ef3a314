"""Builds the CUDA library of evora_b200 in-tree: evora_b200/_lib/libevora_b200.so.

Every translation unit is compiled for sm_100a only.  Per-file flags:
  dropin_strict.cu, fused_f64_strict.cu   --fmad=false (bit-exact FP64 mode)
  fused.cu, gravity.cu, conduction.cu,    --fmad=false (conversions, snapshots, gravity, conduction,
  chem.cu, expansion.cu, grid.cu          floors, expansion terms, the comoving time scalars)
  fused_f32.cu                            --use_fast_math (FP32 form)
Run as `python -m evora_b200.build` (add -v for the ptxas register report).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_lib", "obj")
LIB = os.path.join(LIBDIR, "libevora_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
        "-Xcompiler", "-Wall", "-I", INCLUDE, "-I", CSRC]
PER_FILE = {
    "dropin_strict.cu": ["--fmad=false"],
    "fused_f64_strict.cu": ["--fmad=false"],
    "fused.cu": ["--fmad=false"],
    "gravity.cu": ["--fmad=false"],
    "conduction.cu": ["--fmad=false"],
    "chem.cu": ["--fmad=false"],
    "expansion.cu": ["--fmad=false"],
    "grid.cu": ["--fmad=false"],
    "fused_f32.cu": ["--use_fast_math"],
}
SOURCES = ["abi.cu", "dropin_fast.cu", "dropin_strict.cu", "grid.cu", "fused.cu",
           "fused_f64.cu", "fused_f64_strict.cu", "fused_f32.cu", "batch.cu", "noalloc.cu", "server.cu",
           "io.cu", "gravity.cu", "conduction.cu", "chem.cu", "chem_fast.cu", "expansion.cu"]


def _deps():
    files = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                files.append(os.path.join(d, f))
    return files


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, verbose):
    obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, *BASE, *PER_FILE.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library if any source or header is newer than it."""
    sources = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    os.makedirs(OBJDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(_deps()):
        build_drivers()
        return LIB
    with cf.ThreadPoolExecutor(max_workers=min(8, len(sources))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), sources))
    if verbose:
        for (obj, log), src in zip(results, sources):
            sys.stderr.write(f"== {src}\n{log}")
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    build_drivers()
    return LIB


DRIVERS = {"evora_run": "evora_run.cpp", "evora_post": "evora_post.cpp"}


def build_drivers() -> None:
    """The command-line drivers (csrc/driver/), linked against the library
    with an $ORIGIN run path so that they find it beside themselves."""
    ddir = os.path.join(CSRC, "driver")
    for exe, src in DRIVERS.items():
        out = os.path.join(LIBDIR, exe)
        deps = [os.path.join(ddir, f) for f in os.listdir(ddir)] + [LIB] + _deps()
        if os.path.exists(out) and os.path.getmtime(out) >= _newest(deps):
            continue
        cmd = [NVCC, "-O2", "-std=c++17", "-Xcompiler", "-Wall", "-I", INCLUDE, "-I", CSRC,
               os.path.join(ddir, src), "-o", out + ".tmp", "-L", LIBDIR, "-levora_b200",
               "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed for {src}:\n{r.stdout}\n{r.stderr}")
        os.replace(out + ".tmp", out)


if __name__ == "__main__":
    print(build(force="-f" in sys.argv, verbose="-v" in sys.argv))
