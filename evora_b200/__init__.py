"""evora_b200 -- the hydro update of evora (MUSCL-Hancock predictor and
sweeps, HLL/HLLC fluxes, ghost-cell fill, CFL reduction) as hand-written
CUDA kernels for B200 (sm_100a), behind a C ABI (include/evora_gpu.h)."""
from ._native import LIB_PATH, EvoraError, lib
from .hydro import (CARRY_ENTROPY, FP32, FP32_PAIR_TILE, FP64, REFERENCE_KERNELS, RESIDENT_FP32, RESIDENT_FP64,
                    STRICT, Batch, DropIn, EvoraDerived, EvoraParams, Grid, MultiGrid, default_params, derived,
                    shapes)
from . import ic

__all__ = ["LIB_PATH", "EvoraError", "lib", "Batch", "CARRY_ENTROPY", "FP32", "FP32_PAIR_TILE", "FP64",
           "REFERENCE_KERNELS", "RESIDENT_FP32", "RESIDENT_FP64", "MultiGrid",
           "STRICT", "DropIn", "EvoraDerived", "EvoraParams", "Grid", "default_params", "derived",
           "shapes", "ic"]
