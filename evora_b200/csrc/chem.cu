// chem.cu -- the per-cell step chem(q) of the reference (chemistry.f90:
// 72-121; the cell update in chem_cell.cuh), after the hydro update and
// gravity as main.f90:167 orders it, in the reference's order of operations:
// on a resident SoA state (species in their own FP64 array) for STRICT
// grids, the drop-in chem(q) on the reference layout q(6) or, with
// chemistry, q(12), and coolstep (timestep.f90:106-143) for both.  Species
// and cooling are FP64 whatever the state precision.  This translation unit
// is compiled without FMA contraction; the default mode's chem(q) is in
// chem_fast.cu.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "chem.h"
#include "chem_cell.cuh"
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

// chem(q) on the resident SoA state.  The cooling sub-cycles are a long
// FP64 latency chain per cell (powers, exponentials, divisions): registers
// are capped for 16 warps per SM.
template <typename T>
__global__ void __launch_bounds__(kChemThreads, 4)
k_chem(T* __restrict__ q, int64_t n, int nf, double* __restrict__ species, HydroParams P,
                       const GridCtl* ctl, unsigned* err) {
  if (ctl_skip(ctl)) return;
  chem_soa(q, n, nf, species, P, ctl, CieExact{}, err);
}

// coolstep (timestep.f90:106-143) part 1 on a resident SoA state: the
// smallest cooling time over the cells into ctl->vcool, and the equilibrium
// abundances it computes written back to the species, as the reference's
// call does.  nH, nHe are module global's: the last cell's of the last chem
// (or initchem), whose density nothing has changed since.  T uses the
// pressure primitive() leaves in w(5).
template <typename T>
__global__ void __launch_bounds__(kChemThreads, 4)
k_coolstep(const T* __restrict__ q, int64_t n, int nf, double* __restrict__ species, HydroParams P,
           GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const Gas<double> c = Gas<double>::make(P);
  const Units U = units_of(P, ctl);
  const ChemCoef& k = ctl->coef;
  const double rho_last = (double)q[n - 1];
  const double nH = P.chiH * rho_last, nHe = P.chiHe * rho_last;
  double vmin = 1e6;   // coolstep's initial v
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6], s[kNs];
    load_cell(q, n, nf, i, v);
#pragma unroll
    for (int j = 0; j < kNs; ++j) s[j] = species[j * n + i];
    const double press = pressure(v, c, P.dualenergy != 0, e);
    vmin = fmin2(vmin, cool_time(k, P.background, U.temp0, press, nH, nHe, s, e));
#pragma unroll
    for (int j = 0; j < kNs; ++j) species[j * n + i] = s[j];
  }
  for (int off = 16; off > 0; off >>= 1) vmin = fmin2(vmin, __shfl_xor_sync(0xffffffffu, vmin, off));
  if ((threadIdx.x & 31) == 0) atomicMin(&ctl->vcool, ordered_bits(vmin));
  if (e) atomicOr(&ctl->err, e);
}

// Offset of w(1, ix, iy, iz) in w(5, -1:nx+2, -1:ny+2, -1:nz+2) (0-based
// interior indices).
__device__ __forceinline__ int64_t w_at(const HydroParams& P, int ix, int iy, int iz) {
  return (int64_t)EVORA_NW * (((int64_t)(iz + 2) * (P.ny + 4) + (iy + 2)) * (P.nx + 4) + (ix + 2));
}

// The drop-in coolstep on q(12, cell) and w (ghosts included): out[0] the
// smallest cooling time (ordered bits, preset to 1e6), out[1] the errors.
__global__ void k_coolstep_aos(double* __restrict__ q, const double* __restrict__ w, HydroParams P, ChemCoef k,
                               double nH, double nHe, unsigned long long* out) {
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const Units U = units_of(P, nullptr);
  double vmin = 1e6;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % P.nx);
    const int64_t r = i / P.nx;
    const int iy = (int)(r % P.ny), iz = (int)(r / P.ny);
    const double press = w[w_at(P, ix, iy, iz) + 4];
    double* cell = q + (int64_t)EVORA_NQ_CHEM * i;
    vmin = fmin2(vmin, cool_time(k, P.background, U.temp0, press, nH, nHe, cell + EVORA_NQ, e));
  }
  for (int off = 16; off > 0; off >>= 1) vmin = fmin2(vmin, __shfl_xor_sync(0xffffffffu, vmin, off));
  if ((threadIdx.x & 31) == 0) atomicMin(&out[0], ordered_bits(vmin));
  if (e) atomicOr(reinterpret_cast<unsigned*>(&out[1]), e);
}

// The drop-in on q(nq, cell): nq = 12 with chemistry (n = q(7:12)), else 6.
__global__ void k_chem_aos(double* __restrict__ q, int64_t n, int nq, HydroParams P, ChemCoef k, double dt,
                           unsigned* err) {
  const Gas<double> c = Gas<double>::make(P);
  const Units U = units_of(P, nullptr);
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double* cell = q + (int64_t)nq * i;
    chem_cell(cell, cell + EVORA_NQ, P, U, k, dt, c, CieExact{}, e);
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

int cool_step(const HydroParams& P, const void* q, bool f32, int nf, int64_t n, double* species, GridCtl* ctl,
              cudaStream_t st) {
  const int blocks = (int)((n + kChemThreads - 1) / kChemThreads < 148 * 16 ? (n + kChemThreads - 1) / kChemThreads
                                                                          : 148 * 16);
  if (f32) k_coolstep<float><<<blocks, kChemThreads, 0, st>>>((const float*)q, n, nf, species, P, ctl);
  else k_coolstep<double><<<blocks, kChemThreads, 0, st>>>((const double*)q, n, nf, species, P, ctl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "coolstep");
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
  double* w = nullptr;
  size_t wbytes = 0;
  unsigned* err = nullptr;
  unsigned long long* out = nullptr;   // coolstep: v (ordered bits), errors
};
DropinChem& dchem() {
  static DropinChem s;
  return s;
}
int fail_cuda(cudaError_t e, const char* where) {
  set_cuda_error(e, where);
  return EVORA_ERR_CUDA;
}
void reset_device(DropinChem& D, int dev) {
  if (dev == D.device) return;
  cudaFree(D.q);
  cudaFree(D.w);
  cudaFree(D.err);
  cudaFree(D.out);
  D.q = D.w = nullptr;
  D.err = nullptr;
  D.out = nullptr;
  D.bytes = D.wbytes = 0;
  D.device = dev;
}
// A staging buffer of at least `bytes` for a host array.
cudaError_t stage(double** buf, size_t* have, size_t bytes) {
  if (*have >= bytes) return cudaSuccess;
  cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc(buf, bytes);
  if (e == cudaSuccess) *have = bytes;
  return e;
}
// Module global's nH, nHe after a chem with chemistry: its last cell's.
cudaError_t record_last_cell(const HydroParams& P, const double* q, bool dev_q, int64_t n) {
  double rho = 0.0;
  const double* last = q + (int64_t)EVORA_NQ_CHEM * (n - 1);
  if (dev_q) {
    cudaError_t e = cudaMemcpy(&rho, last, sizeof rho, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
  } else {
    rho = *last;
  }
  dropin_set_nh(P.chiH * rho, P.chiHe * rho);
  return cudaSuccess;
}
}  // namespace

extern "C" int evora_chem(double* q) {
  if (!q) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinChem& D = dchem();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  CosmoTime t;
  ChemCoef k;
  if (!dropin_params(&P) || !dropin_time(&t) || !dropin_coef(&k)) return EVORA_ERR_ARG;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "evora_chem");
  reset_device(D, dev);
  const int nq = P.chemistry ? EVORA_NQ_CHEM : EVORA_NQ;
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const size_t bytes = sizeof(double) * nq * n;
  if (!D.err && (e = cudaMalloc(&D.err, sizeof(unsigned))) != cudaSuccess) return fail_cuda(e, "evora_chem");
  const bool dev_q = is_device_pointer(q);
  double* dq = q;
  if (!dev_q) {
    if ((e = stage(&D.q, &D.bytes, bytes)) != cudaSuccess) return fail_cuda(e, "evora_chem");
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
  // chem sets nH, nHe per cell (chemistry.f90:90-91): the last cell's stay
  if (P.chemistry && (e = record_last_cell(P, q, dev_q, n)) != cudaSuccess) return fail_cuda(e, "evora_chem");
  return (int)herr;
}

extern "C" int evora_coolstep(double* q, const double* w, double* dt) {
  if (!q || !w || !dt) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinChem& D = dchem();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  ChemCoef k;
  double nH, nHe;
  if (!dropin_params(&P) || !dropin_coef(&k) || !dropin_nh(&nH, &nHe)) return EVORA_ERR_ARG;
  if (!P.cooldt || P.noncie) return EVORA_ERR_ARG;   // w(5, ...) of the CIE build
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "evora_coolstep");
  reset_device(D, dev);
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const size_t qbytes = sizeof(double) * EVORA_NQ_CHEM * n;
  const size_t wbytes = sizeof(double) * EVORA_NW * (P.nx + 4) * (P.ny + 4) * (P.nz + 4);
  if (!D.out && (e = cudaMalloc(&D.out, 2 * sizeof(unsigned long long))) != cudaSuccess)
    return fail_cuda(e, "evora_coolstep");
  const bool dev_q = is_device_pointer(q);
  double* dq = q;
  const double* dw = w;
  if (!dev_q) {
    if ((e = stage(&D.q, &D.bytes, qbytes)) != cudaSuccess ||
        (e = cudaMemcpy(D.q, q, qbytes, cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail_cuda(e, "evora_coolstep");
    dq = D.q;
  }
  if (!is_device_pointer(w)) {
    if ((e = stage(&D.w, &D.wbytes, wbytes)) != cudaSuccess ||
        (e = cudaMemcpy(D.w, w, wbytes, cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail_cuda(e, "evora_coolstep");
    dw = D.w;
  }
  const double big = 1e6;   // coolstep's initial v
  unsigned long long init[2] = {0ull, 0ull};
  std::memcpy(&init[0], &big, sizeof big);
  if ((e = cudaMemcpy(D.out, init, sizeof init, cudaMemcpyHostToDevice)) != cudaSuccess)
    return fail_cuda(e, "evora_coolstep");
  k_coolstep_aos<<<grid_of(n), kThreads>>>(dq, dw, P, k, nH, nHe, D.out);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
    return fail_cuda(e, "evora_coolstep");
  unsigned long long out[2];
  if ((e = cudaMemcpy(out, D.out, sizeof out, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_coolstep");
  if (!dev_q && (e = cudaMemcpy(q, dq, qbytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_coolstep");
  unsigned err = (unsigned)out[1];
  if (err) return (int)err;
  double v;
  std::memcpy(&v, &out[0], sizeof v);
  *dt = cool_dt(P.c_cooldt, v, *dt, err);
  return (int)err;
}
