// expansion.h -- the expansion terms of comoving runs for resident grids.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

// expansion(q), cosmology.f90:53-72: pressure() (dual-energy write-back),
// then E -= dt (3g-5) expand p / (g-1) and S -= dt (3g-5) expand S, in place
// on a SoA state (nf fields, f32 or f64) with dt and expand from ctl; errors
// of pressure() go to ctl->err.
int expansion_step(const HydroParams& P, void* q, bool f32, int nf, int64_t n, GridCtl* ctl, cudaStream_t st);

}  // namespace evora
