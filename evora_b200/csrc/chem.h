// chem.h -- the chem(q) step (pressure floors; with the CIE build, the
// equilibrium species and the cooling) for resident grids.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

// chem(q), chemistry.f90:72-121, in place on a SoA state (nf fields, f32 or
// f64) and, with chemistry, its FP64 species (6 field-major arrays of n
// cells); dt and the rate coefficients from ctl; errors go to ctl->err.
int chem_step(const HydroParams& P, void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
              cudaStream_t st);

// The same on a grid of the default mode: fewer FP64 operations per cooling
// sub-cycle (shared powers of T, a table-driven exponential, contracted
// products), within a few ulp of chem_step per rate (chem_fast.cu).  With
// expand, each cell then takes the expansion terms of a comoving run
// (expansion(q), cosmology.f90:53-72) in the same pass.
int chem_step_fast(const HydroParams& P, void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
                   cudaStream_t st, bool expand = false);

// coolstep (timestep.f90:106-143) part 1 on the state at the start of a
// step (nf fields, f32 or f64) and its species: the smallest cooling time
// into ctl->vcool (preset by the step's first kernel), the equilibrium
// abundances written back to the species as the reference's call does.
int cool_step(const HydroParams& P, const void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
              cudaStream_t st);

// The rate coefficients at the start of a run (initchem's compcoef, uv = 0)
// and after a comoving step's compunits (compbackground, compcoef).
void start_coef(const HydroParams& P, double cosmo, ChemCoef* k);
void step_coef(const HydroParams& P, double cosmo, double redshift, ChemCoef* k);

}  // namespace evora
