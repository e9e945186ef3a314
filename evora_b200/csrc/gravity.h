// gravity.h -- self-gravity of the hydro state on the device:
// gravitation.f90 (gravpotential with both source terms, multigreen,
// gravintegration, grav_force) with cuFFT.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include "hydro_math.cuh"

namespace evora {

// Constants of compparameter that the Poisson solve reads
// (parameter.f90:219-264) and the device buffers of one grid's solve.
struct GravPlan {
  int nx = 0, ny = 0, nz = 0;
  int64_t n = 0;          // cells
  int64_t nh = 0;         // complex coefficients of the half spectrum
  bool comoving = false;  // source cosmo grav (rho / fb - 1) (gravitation.f90:36-37)
  double grav = 0.0;      // 4 pi G (global.f90:101), or 1.5 omega0 when comoving
  double fb = 1.0;
  double dx2inv = 0.0, dy2inv = 0.0, dz2inv = 0.0;   // 0.5 / dx ...
  cufftHandle fwd = 0, inv = 0;                       // D2Z, Z2D over (nz, ny, nx)
  double* phi = nullptr;                              // potential, n (real)
  cufftDoubleComplex* spec = nullptr;                 // its spectrum, nh
  double* green = nullptr;    // sin^2 tables of multigreen: nx + ny + nz
  double* red = nullptr;      // partial sums of rho and the mean (device)
  int nred = 0;
  double h2 = 0.0;            // dx^2 / 4
  cudaStream_t stream = nullptr;
  bool ready = false;
};

// Builds the plans and buffers for a grid (cufftPlan3d on stream `st`).
// Returns 0, EVORA_ERR_NOMEM or EVORA_ERR_CUDA.
int grav_plan(const HydroParams& P, GravPlan* g, cudaStream_t st);
void grav_plan_free(GravPlan* g);
void grav_set_stream(GravPlan* g, cudaStream_t st);

// gravpotential (gravitation.f90:26-53): phi from the density of the state
// (SoA with nf fields of type f32 or f64, or the reference AoS q(6, n)); the
// comoving source takes cosmo from ctl, or cosmo_host when ctl is null.
int grav_potential(GravPlan& g, const void* q, bool f32, int nf, int aos, const GridCtl* ctl, double cosmo_host);

// gravintegration (gravitation.f90:170-194) with the forces of grav_force
// (196-243), in place on the state, with the step's dt from ctl (or dt_host
// when ctl is null).  With `expand` (a grid's parameters; SoA state and ctl
// required) the comoving step's expansion terms (cosmology.f90:53-72) are
// applied to each cell in the same pass.
int grav_integrate(GravPlan& g, void* q, bool f32, int nf, int aos, const GridCtl* ctl, double dt_host,
                   const HydroParams* expand = nullptr);

}  // namespace evora
