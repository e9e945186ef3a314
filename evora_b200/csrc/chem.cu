// chem.cu -- the per-cell step chem(q) of the reference (chemistry.f90:
// 72-121) in the plain build (no chemical species): pressure() with its
// dual-energy write-back, then the temperature and Jeans pressure floors
//
//   press = max(press, temp_fl rho temp0inv)        (tempfloor, temp2press)
//   press = max(press, jeansfloor0 rho rho)          (jeansfloor)
//   E += dpress / (g-1),  S += dpress / rho^(g-1)
//
// on a resident SoA state after the hydro update and gravity, as main.f90:167
// orders it; plus the drop-in chem(q) on the reference layout.  This
// translation unit is compiled without FMA contraction.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "chem.h"
#include "common.h"

namespace evora {
namespace {

constexpr int kThreads = 256;

int grid_of(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

// One cell: v holds q(1:6) in FP64 (in place); temp0inv of the step's units.
__device__ __forceinline__ void floor_cell(double* v, const HydroParams& P, double temp0inv, const Gas<double>& c,
                                           unsigned& err) {
  double press = pressure(v, c, P.dualenergy != 0, err);
  const double oldpress = press;
  if (P.tempfloor) {
    const double pfloor = P.temp_fl * v[0] * temp0inv;     // temp2press, comp.f90:104-119
    if (pfloor > press) press = pfloor;                     // max(press, pfloor)
  }
  if (P.jeansfloor) {
    const double pfloor = P.jeansfloor0 * v[0] * v[0];
    if (pfloor > press) press = pfloor;
  }
  const double dpress = press - oldpress;
  v[4] = v[4] + dpress * P.g1inv;
  v[5] = v[5] + dpress / pow(v[0], P.g1);
}

template <typename T>
__global__ void k_floors(T* __restrict__ q, int64_t n, int nf, HydroParams P, const GridCtl* ctl, unsigned* err) {
  if (ctl_skip(ctl)) return;
  const Gas<double> c = Gas<double>::make(P);
  const double temp0inv = units_of(P, ctl).temp0inv;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6];
    load_cell(q, n, nf, i, v);   // S not carried (nf = 5): the S terms are dropped
    floor_cell(v, P, temp0inv, c, e);
    q[4 * n + i] = (T)v[4];
    if (nf == 6) q[5 * n + i] = (T)v[5];
  }
  if (e) atomicOr(err, e);
}

__global__ void k_floors_aos(double* __restrict__ q, int64_t n, HydroParams P, unsigned* err) {
  const Gas<double> c = Gas<double>::make(P);
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    floor_cell(q + (int64_t)EVORA_NQ * i, P, P.temp0inv, c, e);
  if (e) atomicOr(err, e);
}

}  // namespace

int chem_floors(const HydroParams& P, void* q, bool f32, int nf, int64_t n, GridCtl* ctl, cudaStream_t st) {
  if (f32) k_floors<float><<<grid_of(n), kThreads, 0, st>>>((float*)q, n, nf, P, ctl, &ctl->err);
  else k_floors<double><<<grid_of(n), kThreads, 0, st>>>((double*)q, n, nf, P, ctl, &ctl->err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "chem");
    return EVORA_ERR_CUDA;
  }
  return 0;
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
  if (!dropin_params(&P)) return EVORA_ERR_ARG;
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
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const size_t bytes = sizeof(double) * EVORA_NQ * n;
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
  k_floors_aos<<<grid_of(n), kThreads>>>(dq, n, P, D.err);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  unsigned herr = 0;
  if ((e = cudaMemcpy(&herr, D.err, sizeof herr, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  if (!dev_q && (e = cudaMemcpy(q, dq, bytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return fail_cuda(e, "evora_chem");
  return (int)herr;
}
