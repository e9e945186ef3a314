// chem.h -- the plain-build chem(q) step (pressure floors) for resident grids.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

// chem(q), chemistry.f90:72-121, without species: pressure() (dual-energy
// write-back), the temperature and Jeans floors and the E and S
// corrections, in place on a SoA state (nf fields, f32 or f64); errors of
// pressure() go to ctl->err.
int chem_floors(const HydroParams& P, void* q, bool f32, int nf, int64_t n, GridCtl* ctl, cudaStream_t st);

}  // namespace evora
