// expansion.cu -- the adiabatic expansion terms of a comoving run
// (expansion(q), cosmology.f90:53-72), which main.f90:178 applies after the
// hydro update, gravity, chem and conduction when supercomoving and not
// atomic:
//
//   press = pressure(q)                     (comp.f90:45-85, write-back)
//   E = E - dt * g35 * expand * press / g1
//   S = S - dt * g35 * expand * S
//
// with g35 = 3g - 5 and expand = a da/dt of the step's compcosmo, both
// products associated left to right as there.  One pass over the resident
// SoA state, and the drop-in on the reference layout.  This translation unit
// is compiled without FMA contraction.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "common.h"
#include "cosmology.cuh"
#include "expansion.h"

namespace evora {
namespace {

constexpr int kThreads = 256;

int grid_of(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

// One cell: v holds q(1:6) in FP64 (in place); k = dt * g35 * expand.
__device__ __forceinline__ void expand_cell(double* v, double k, const HydroParams& P, const Gas<double>& c,
                                            unsigned& err) {
  const double press = pressure(v, c, P.dualenergy != 0, err);
  v[4] = v[4] - k * press / P.g1;
  v[5] = v[5] - k * v[5];
}

template <typename T>
__global__ void k_expansion(T* __restrict__ q, int64_t n, int nf, HydroParams P, const GridCtl* ctl, unsigned* err) {
  if (ctl_skip(ctl)) return;
  const Gas<double> c = Gas<double>::make(P);
  const double k = ctl->dt * P.g35 * ctl->expand;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6];
    load_cell(q, n, nf, i, v);   // S not carried (nf = 5): it never feeds back without dual energy
    expand_cell(v, k, P, c, e);
    q[4 * n + i] = (T)v[4];
    if (nf == 6) q[5 * n + i] = (T)v[5];
  }
  if (e) atomicOr(err, e);
}

__global__ void k_expansion_aos(double* __restrict__ q, int64_t n, HydroParams P, double dt, double expand,
                                unsigned* err) {
  const Gas<double> c = Gas<double>::make(P);
  const double k = dt * P.g35 * expand;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    expand_cell(q + (int64_t)EVORA_NQ * i, k, P, c, e);
  if (e) atomicOr(err, e);
}

}  // namespace

int expansion_step(const HydroParams& P, void* q, bool f32, int nf, int64_t n, GridCtl* ctl, cudaStream_t st) {
  if (f32) k_expansion<float><<<grid_of(n), kThreads, 0, st>>>((float*)q, n, nf, P, ctl, &ctl->err);
  else k_expansion<double><<<grid_of(n), kThreads, 0, st>>>((double*)q, n, nf, P, ctl, &ctl->err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "expansion");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

}  // namespace evora

using namespace evora;

namespace {
struct DropinExpansion {
  std::mutex mu;
  int device = -1;
  double* q = nullptr;
  size_t bytes = 0;
  unsigned* err = nullptr;
};
DropinExpansion& dexp() {
  static DropinExpansion s;
  return s;
}
int fail_cuda(cudaError_t e, const char* where) {
  set_cuda_error(e, where);
  return EVORA_ERR_CUDA;
}
}  // namespace

extern "C" int evora_expansion(double* q) {
  if (!q) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinExpansion& D = dexp();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  CosmoTime s;
  if (!dropin_params(&P) || !dropin_time(&s)) return EVORA_ERR_ARG;
  if (P.chemistry) return EVORA_ERR_ARG;   // the drop-in reads q(6, ...); grids take q(12, ...)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "evora_expansion");
  if (dev != D.device) {
    cudaFree(D.q);
    cudaFree(D.err);
    D.q = nullptr;
    D.err = nullptr;
    D.bytes = 0;
    D.device = dev;
  }
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const size_t bytes = sizeof(double) * EVORA_NQ * n;
  if (!D.err && (e = cudaMalloc(&D.err, sizeof(unsigned))) != cudaSuccess) return fail_cuda(e, "evora_expansion");
  const bool dev_q = is_device_pointer(q);
  double* dq = q;
  if (!dev_q) {
    if (D.bytes < bytes) {
      cudaFree(D.q);
      D.q = nullptr;
      D.bytes = 0;
      if ((e = cudaMalloc(&D.q, bytes)) != cudaSuccess) return fail_cuda(e, "evora_expansion");
      D.bytes = bytes;
    }
    if ((e = cudaMemcpy(D.q, q, bytes, cudaMemcpyHostToDevice)) != cudaSuccess) return fail_cuda(e, "evora_expansion");
    dq = D.q;
  }
  if ((e = cudaMemset(D.err, 0, sizeof(unsigned))) != cudaSuccess) return fail_cuda(e, "evora_expansion");
  k_expansion_aos<<<grid_of(n), kThreads>>>(dq, n, P, s.dt, s.expand, D.err);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
    return fail_cuda(e, "evora_expansion");
  unsigned herr = 0;
  if ((e = cudaMemcpy(&herr, D.err, sizeof herr, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_expansion");
  if (!dev_q && (e = cudaMemcpy(q, dq, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_expansion");
  return (int)herr;
}
