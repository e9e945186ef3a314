// noalloc.cu -- evora_hydrostep_noalloc: the CFL time step of hydrostep
// (timestep.f90:26-57) for callers that must not allocate device memory.
//
// Who needs it: a driver that allocates all of its device memory once at
// start-up and may not allocate inside its time loop (the reference's own
// driver allocates q, w, evo, s once, main.f90:72-75); code running while a
// memory pool owns the device or while other work is being captured, where a
// cudaMalloc would fail, synchronise the device or be forbidden by policy.
// evora_hydrostep gets its reduction scratch from cudaMalloc (once, on its
// first call); this variant keeps the scratch in a fixed file-scope device
// array instead and calls no allocating routine.
//
// The scratch: g_hydrostep_scratch, 256-byte aligned, holds one partial
// maximum per axis for every 256-cell block of the grid, then the result.
// Its size caps the grid at kMaxCells interior cells; larger grids are
// rejected with EVORA_ERR_ARG.  Every GPU that loads the library keeps this
// array (about 1.5 MB) until the process exits.  All calls share it, so
// calls that overlap on the GPU (several host threads, or several streams)
// race on it; calls on one stream in sequence are safe.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "common.h"

namespace {

constexpr int kBlock = 256;
constexpr int64_t kMaxCells = int64_t(1) << 24;                 // 256^3 interior cells
constexpr int kMaxBlocks = (int)(kMaxCells / kBlock);           // 65536
constexpr int kSlotDt = 3 * kMaxBlocks;                        // result dt (double bits)
constexpr int kSlotErr = kSlotDt + 1;                          // error mask
constexpr int kScratchWords = kSlotErr + 1;
constexpr int kMaxDevices = 64;

// [0, 3*kMaxBlocks): per-block maxima of |u|+a, |v|+a, |w|+a (double bits);
// [kSlotDt]: dt; [kSlotErr]: EVORA_ERR_* mask.
static __device__ __align__(256) unsigned long long g_hydrostep_scratch[kScratchWords];

// Part 1: one block per 256 interior cells writes its three maxima.  Every
// slot the finisher reads is written by the same call, so nothing needs
// clearing between calls.
__global__ void __launch_bounds__(kBlock) k_partial_max(evora::HydroParams P, const double* __restrict__ w,
                                                       unsigned long long* scratch, int64_t n) {
  const int64_t idx = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  if (idx < n) {
    const int i = (int)(idx % P.nx) + 1;
    const int j = (int)((idx / P.nx) % P.ny) + 1;
    const int k = (int)(idx / ((int64_t)P.nx * P.ny)) + 1;
    const int64_t off = (int64_t)EVORA_NW *
                        ((int64_t)(i + 1) + (int64_t)(P.nx + 4) * ((int64_t)(j + 1) + (int64_t)(P.ny + 4) * (k + 1)));
    const double* c = w + off;
    const double a = sqrt(P.g * c[4] / c[0]);     // timestep.f90:40
    const double s0 = fabs(c[1]) + a, s1 = fabs(c[2]) + a, s2 = fabs(c[3]) + a;
    if (s0 > m0) m0 = s0;                          // NaN speeds are skipped
    if (s1 > m1) m1 = s1;
    if (s2 > m2) m2 = s2;
  }
  __shared__ double red[3][kBlock];
  red[0][threadIdx.x] = m0;
  red[1][threadIdx.x] = m1;
  red[2][threadIdx.x] = m2;
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int d = 0; d < 3; ++d) red[d][threadIdx.x] = evora::fmax2(red[d][threadIdx.x], red[d][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d)
      scratch[3 * blockIdx.x + d] = (unsigned long long)__double_as_longlong(red[d][0]);
}

// Part 2: one block reduces the partial maxima and forms dt (cfl_dt).
__global__ void __launch_bounds__(1024) k_finish(evora::HydroParams P, unsigned long long* scratch, int nb,
                                                 double dt_in) {
  double m[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    for (int d = 0; d < 3; ++d) m[d] = evora::fmax2(m[d], __longlong_as_double((long long)scratch[3 * b + d]));
  __shared__ double red[3][1024];
  for (int d = 0; d < 3; ++d) red[d][threadIdx.x] = m[d];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int d = 0; d < 3; ++d) red[d][threadIdx.x] = evora::fmax2(red[d][threadIdx.x], red[d][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    unsigned e = 0;
    const double dt = evora::cfl_dt(P, red[0][0], red[1][0], red[2][0], dt_in, e);
    scratch[kSlotDt] = (unsigned long long)__double_as_longlong(dt);
    scratch[kSlotErr] = e;
  }
}

std::mutex g_mu;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

// Device address of g_hydrostep_scratch on the current device, looked up
// once per device (with that device current) and cached.
int scratch_address(unsigned long long** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    evora::set_cuda_error(e, "evora_hydrostep_noalloc: cudaGetDevice");
    return EVORA_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    evora::set_error_message("evora_hydrostep_noalloc: device ordinal out of range");
    return EVORA_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_hydrostep_scratch);
    if (e != cudaSuccess || !p) {
      evora::set_cuda_error(e, "evora_hydrostep_noalloc: cudaGetSymbolAddress");
      return EVORA_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned long long*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace

extern "C" int evora_hydrostep_noalloc(const double* w, double* dt) {
  if (!w || !dt) return EVORA_ERR_ARG;
  evora::HydroParams P;
  if (!evora::dropin_params(&P)) {
    evora::set_error_message("evora_hydrostep_noalloc: call evora_set_params first");
    return EVORA_ERR_ARG;
  }
  if (P.noncie) {
    evora::set_error_message("evora_hydrostep_noalloc: w has 11 primitives in the non-equilibrium build");
    return EVORA_ERR_ARG;
  }
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  if (n > kMaxCells) {
    char msg[160];
    std::snprintf(msg, sizeof msg,
                  "evora_hydrostep_noalloc: %lld interior cells exceed the maximum of %lld",
                  (long long)n, (long long)kMaxCells);
    evora::set_error_message(msg);
    return EVORA_ERR_ARG;
  }
  if (!evora::is_device_pointer(w)) {
    evora::set_error_message("evora_hydrostep_noalloc: w must be device memory (no staging copy is made)");
    return EVORA_ERR_ARG;
  }
  unsigned long long* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  const int nb = (int)((n + kBlock - 1) / kBlock);
  k_partial_max<<<nb, kBlock>>>(P, w, scratch, n);
  k_finish<<<1, 1024>>>(P, scratch, nb, *dt);
  // a launch that failed would leave the previous call's dt in the array
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    evora::set_cuda_error(e, "evora_hydrostep_noalloc: launch");
    return EVORA_ERR_CUDA;
  }
  unsigned long long res[2];
  e = cudaMemcpy(res, scratch + kSlotDt, sizeof res, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    evora::set_cuda_error(e, "evora_hydrostep_noalloc");
    return EVORA_ERR_CUDA;
  }
  std::memcpy(dt, &res[0], sizeof(double));   // as evora_hydrostep: dt is set, then the status
  return (int)(unsigned)res[1];
}
