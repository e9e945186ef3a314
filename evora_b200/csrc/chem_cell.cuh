// chem_cell.cuh -- one cell of chem(q) (chemistry.f90:72-121) and the
// per-cell loop of the resident SoA kernel, shared by the reference-order
// kernels (chem.cu, compiled without FMA contraction) and the reduced-work
// ones of the default mode (chem_fast.cu).  The CIE update is a policy:
// Cie::run(C, k, temp0, dt, rho, press, n, err) does cie (cie.f90:26-56).
//
//   press = pressure(q)                              (dual-energy write-back)
//   with chemistry: n in ionisation equilibrium at (rho, press) and, with
//     cooling, press advanced over dt by the sub-cycled cooling update
//     (cie); the non-equilibrium build's ncie (ncie.f90:26-90)
//   press = max(press, temp2press(temp_fl))          (tempfloor)
//   press = max(press, jeansfloor0 rho rho)          (jeansfloor)
//   E += dpress / (g-1),  S += dpress / rho^(g-1)   (cooling or a floor)
#pragma once

#include <cstdint>

#include "chemistry.cuh"
#include "hydro_math.cuh"

namespace evora {

// One cell: v holds q(1:6) in FP64 (in place), n the species (in place;
// read only with chemistry); U the step's units, k its rate coefficients.
// The policy also gives pressure() (comp.f90:45-85) and the power rho^(g-1).
template <class Cie>
__device__ __forceinline__ void chem_cell(double* v, double* n, const HydroParams& P, const Units& U,
                                          const ChemCoef& k, double dt, const Gas<double>& c, const Cie& cie_fn,
                                          unsigned& err) {
  double press = cie_fn.pressure(v, c, P.dualenergy != 0, err);
  const double oldpress = press;
  if (P.chemistry) {
    const ChemParams C{P.cooling, P.background, P.chiH, P.chiHe, P.c_chem, P.substep};
    if (P.noncie) ncie(C, k, U.temp0, dt, press, n, err);
    else cie_fn.run(C, k, U.temp0, dt, v[0], press, n, err);
  }
  if (P.cooling || P.tempfloor || P.jeansfloor) {
    if (P.tempfloor) {
      // temp2press (comp.f90:104-119): temp sum(n) temp0inv with chemistry,
      // temp rho temp0inv without
      const double pfloor = P.chemistry ? P.temp_fl * nsum(n) * U.temp0inv : P.temp_fl * v[0] * U.temp0inv;
      if (pfloor > press) press = pfloor;   // max(press, pfloor)
    }
    if (P.jeansfloor) {
      const double pfloor = P.jeansfloor0 * v[0] * v[0];
      if (pfloor > press) press = pfloor;
    }
    const double dpress = press - oldpress;
    v[4] = v[4] + dpress * P.g1inv;
    v[5] = v[5] + cie_fn.div_pow(dpress, v[0], P.g1);
  }
}

// The expansion terms of a comoving run (expansion(q), cosmology.f90:53-72)
// on the same cell, kx = dt g35 expand: press = pressure(q) (write-back),
// E -= kx press / g1, S -= kx S.
template <class Cie>
__device__ __forceinline__ void expand_cell_t(double* v, double kx, const HydroParams& P, const Gas<double>& c,
                                              const Cie& cie_fn, unsigned& err) {
  const double press = cie_fn.pressure(v, c, P.dualenergy != 0, err);
  v[4] = v[4] - cie_fn.div(kx * press, P.g1, P.g1inv);
  v[5] = v[5] - kx * v[5];
}

// chem(q) over the cells of a SoA state q (nf fields of n cells, T = float
// or double) with its FP64 species (kNs field-major arrays), grid-stride;
// errors OR-ed into *err.  S (field 5) is not carried when nf = 5: its
// terms are dropped.  expand: the expansion terms follow on each cell
// (main.f90:178 runs them right after chem when there is no conduction).
template <typename T, class Cie>
__device__ __forceinline__ void chem_soa(T* __restrict__ q, int64_t n, int nf, double* __restrict__ species,
                                         const HydroParams& P, const GridCtl* ctl, const Cie& cie_fn,
                                         unsigned* err, bool expand = false) {
  const Gas<double> c = Gas<double>::make(P);
  const Units U = units_of(P, ctl);
  const ChemCoef& k = ctl->coef;
  const double dt = ctl->dt;
  const double kx = dt * P.g35 * ctl->expand;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6], s[kNs];
    load_cell(q, n, nf, i, v);
    if (P.chemistry)
#pragma unroll
      for (int j = 0; j < kNs; ++j) s[j] = species[j * n + i];
    chem_cell(v, s, P, U, k, dt, c, cie_fn, e);
    if (expand) expand_cell_t(v, kx, P, c, cie_fn, e);
    q[4 * n + i] = (T)v[4];
    if (nf == 6) q[5 * n + i] = (T)v[5];
    if (P.chemistry)
#pragma unroll
      for (int j = 0; j < kNs; ++j) species[j * n + i] = s[j];
  }
  if (e) atomicOr(err, e);
}

// cie in the reference's order of operations (chemistry.cuh), the
// library's pressure() and pow, and divisions.
struct CieExact {
  __device__ __forceinline__ void run(const ChemParams& C, const ChemCoef& k, double temp0, double dt, double rho,
                                      double& press, double* n, unsigned& err) const {
    cie(C, k, temp0, dt, rho, press, n, err);
  }
  __device__ __forceinline__ double pressure(double* v, const Gas<double>& c, bool de, unsigned& err) const {
    return evora::pressure(v, c, de, err);
  }
  // a / x^y
  __device__ __forceinline__ double div_pow(double a, double x, double y) const { return a / pow(x, y); }
  // a / b (binv = 1/b rounded, unused)
  __device__ __forceinline__ double div(double a, double b, double) const { return a / b; }
};

}  // namespace evora
