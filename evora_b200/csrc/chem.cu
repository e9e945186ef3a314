// chem.cu -- the per-cell step chem(q) of the reference (chemistry.f90:
// 72-121), after the hydro update and gravity as main.f90:167 orders it:
//
//   press = pressure(q)                              (dual-energy write-back)
//   with chemistry (CIE build): n = q(7:12) in ionisation equilibrium at
//     (rho, press) and, with cooling, press advanced over dt by the
//     sub-cycled cooling update (cie, cie.f90:26-56; chemistry.cuh)
//   press = max(press, temp2press(temp_fl))          (tempfloor)
//   press = max(press, jeansfloor0 rho rho)          (jeansfloor)
//   E += dpress / (g-1),  S += dpress / rho^(g-1)   (cooling or a floor)
//
// on a resident SoA state (species in their own FP64 array), plus the
// drop-in chem(q) on the reference layout q(6) or, with chemistry, q(12).
// Species and cooling are FP64 whatever the state precision.  This
// translation unit is compiled without FMA contraction.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "chem.h"
#include "chemistry.cuh"
#include "common.h"

namespace evora {
namespace {

constexpr int kThreads = 256;
constexpr int kChemThreads = 128;

int grid_of(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

// One cell: v holds q(1:6) in FP64 (in place), n the species (in place;
// read only with chemistry); U the step's units, k its rate coefficients.
__device__ __forceinline__ void chem_cell(double* v, double* n, const HydroParams& P, const Units& U,
                                          const ChemCoef& k, double dt, const Gas<double>& c, unsigned& err) {
  double press = pressure(v, c, P.dualenergy != 0, err);
  const double oldpress = press;
  if (P.chemistry) {
    const ChemParams C{P.cooling, P.background, P.chiH, P.chiHe, P.c_chem, P.substep};
    cie(C, k, U.temp0, dt, v[0], press, n, err);
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
    v[5] = v[5] + dpress / pow(v[0], P.g1);
  }
}

// The cooling sub-cycles are a long FP64 latency chain per cell (powers,
// exponentials, divisions): registers are capped for 16 warps per SM.
template <typename T>
__global__ void __launch_bounds__(kChemThreads, 4)
k_chem(T* __restrict__ q, int64_t n, int nf, double* __restrict__ species, HydroParams P,
                       const GridCtl* ctl, unsigned* err) {
  if (ctl_skip(ctl)) return;
  const Gas<double> c = Gas<double>::make(P);
  const Units U = units_of(P, ctl);
  const ChemCoef& k = ctl->coef;
  const double dt = ctl->dt;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6], s[kNs];
    load_cell(q, n, nf, i, v);   // S not carried (nf = 5): the S terms are dropped
    if (P.chemistry)
#pragma unroll
      for (int j = 0; j < kNs; ++j) s[j] = species[j * n + i];
    chem_cell(v, s, P, U, k, dt, c, e);
    q[4 * n + i] = (T)v[4];
    if (nf == 6) q[5 * n + i] = (T)v[5];
    if (P.chemistry)
#pragma unroll
      for (int j = 0; j < kNs; ++j) species[j * n + i] = s[j];
  }
  if (e) atomicOr(err, e);
}

// The drop-in on q(nq, cell): nq = 12 with chemistry (n = q(7:12)), else 6.
__global__ void k_chem_aos(double* __restrict__ q, int64_t n, int nq, HydroParams P, ChemCoef k, double dt,
                           unsigned* err) {
  const Gas<double> c = Gas<double>::make(P);
  const Units U = units_of(P, nullptr);
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double* cell = q + (int64_t)nq * i;
    chem_cell(cell, cell + EVORA_NQ, P, U, k, dt, c, e);
  }
  if (e) atomicOr(err, e);
}

}  // namespace

int chem_step(const HydroParams& P, void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
              cudaStream_t st) {
  const int blocks = (int)((n + kChemThreads - 1) / kChemThreads < 148 * 16 ? (n + kChemThreads - 1) / kChemThreads
                                                                          : 148 * 16);
  if (f32) k_chem<float><<<blocks, kChemThreads, 0, st>>>((float*)q, n, nf, species, P, ctl, &ctl->err);
  else k_chem<double><<<blocks, kChemThreads, 0, st>>>((double*)q, n, nf, species, P, ctl, &ctl->err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "chem");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

void start_coef(const HydroParams& P, double cosmo, ChemCoef* k) {
  // initchem's compcoef (chemistry.f90:38) at the start of the run, before
  // any compbackground: uv = 0 (main.f90:94, 134)
  compcoef(chem_units(P, cosmo), 0.0, *k);
}

void step_coef(const HydroParams& P, double cosmo, double redshift, ChemCoef* k) {
  // compbackground and compcoef after compunits (main.f90:134-135)
  const double uv = compbackground(P.background, P.bg, P.j0, redshift, cosmo, k->uv);
  compcoef(chem_units(P, cosmo), uv, *k);
}

}  // namespace evora

using namespace evora;

namespace {
struct DropinChem {
  std::mutex mu;
  int device = -1;
  double* q = nullptr;
  size_t bytes = 0;
  unsigned* err = nullptr;
};
DropinChem& dchem() {
  static DropinChem s;
  return s;
}
int fail_cuda(cudaError_t e, const char* where) {
  set_cuda_error(e, where);
  return EVORA_ERR_CUDA;
}
}  // namespace

extern "C" int evora_chem(double* q) {
  if (!q) return EVORA_ERR_ARG;
  DropinChem& D = dchem();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  CosmoTime t;
  ChemCoef k;
  if (!dropin_params(&P) || !dropin_time(&t) || !dropin_coef(&k)) return EVORA_ERR_ARG;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "evora_chem");
  if (dev != D.device) {
    cudaFree(D.q);
    cudaFree(D.err);
    D.q = nullptr;
    D.err = nullptr;
    D.bytes = 0;
    D.device = dev;
  }
  const int nq = P.chemistry ? EVORA_NQ_CHEM : EVORA_NQ;
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const size_t bytes = sizeof(double) * nq * n;
  if (!D.err && (e = cudaMalloc(&D.err, sizeof(unsigned))) != cudaSuccess) return fail_cuda(e, "evora_chem");
  const bool dev_q = is_device_pointer(q);
  double* dq = q;
  if (!dev_q) {
    if (D.bytes < bytes) {
      cudaFree(D.q);
      D.q = nullptr;
      D.bytes = 0;
      if ((e = cudaMalloc(&D.q, bytes)) != cudaSuccess) return fail_cuda(e, "evora_chem");
      D.bytes = bytes;
    }
    if ((e = cudaMemcpy(D.q, q, bytes, cudaMemcpyHostToDevice)) != cudaSuccess) return fail_cuda(e, "evora_chem");
    dq = D.q;
  }
  if ((e = cudaMemset(D.err, 0, sizeof(unsigned))) != cudaSuccess) return fail_cuda(e, "evora_chem");
  k_chem_aos<<<grid_of(n), kThreads>>>(dq, n, nq, P, k, t.dt, D.err);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  unsigned herr = 0;
  if ((e = cudaMemcpy(&herr, D.err, sizeof herr, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  if (!dev_q && (e = cudaMemcpy(q, dq, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  return (int)herr;
}
