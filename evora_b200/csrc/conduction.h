// conduction.h -- explicit thermal conduction (conduction.f90) for resident
// grids, and its time-step limit (thermalstep, timestep.f90:72-104).
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

struct CondPlan {
  int64_t n = 0;
  double* temp = nullptr;   // T = p / rho * temp0 per cell (FP64)
};

int cond_plan(int64_t n, CondPlan* c);
void cond_plan_free(CondPlan* c);

// primitive + thermalconduction on a SoA state (nf fields, f32 or f64), in
// place, with dt from ctl (dt_host when ctl is null; errors of pressure()
// go to ctl->err).
int cond_step(CondPlan& c, const HydroParams& P, void* q, bool f32, int nf, GridCtl* ctl, double dt_host,
              cudaStream_t st);

// thermalstep per cell: rho / kappa with kappa = kappa0 T^2.5, T from
// pressure() (no write-back) over rho times temp0 (U: the step's units).
__host__ __device__ inline double thermal_v(const Units& U, double rho, double press) {
  const double temp = press / rho * U.temp0;
  const double kappa = U.kappa0 * pow(temp, 2.5);
  return rho / kappa;
}

// The same with T^2.5 = T^2 sqrt(T) (within a few ulp of pow; the fast
// arithmetic forms use it, the strict form keeps pow).
__host__ __device__ inline double thermal_v_fast(const Units& U, double rho, double press) {
  const double temp = press / rho * U.temp0;
  const double kappa = U.kappa0 * (temp * temp * sqrt(temp));
  return rho / kappa;
}

// thermalstep part 2: dt = min(c_cond dx^2 vmin / temp0, dt); EVORA_ERR_DT if <= 0.
__host__ __device__ inline double thermal_dt(const HydroParams& P, const Units& U, double vmin, double dt,
                                             unsigned& err) {
  const double v = P.c_cond * (P.dx * P.dx) * vmin / U.temp0;
  const double d = (dt < v) ? dt : v;
  if (d <= 0.0) err |= EVORA_ERR_DT;
  return d;
}

}  // namespace evora
