// conduction.cu -- explicit thermal conduction on the device, the reference's
// conduction.f90 for a resident grid:
//
//   after the hydro update (main.f90:169-175): primitive (with its dual-
//   energy write-back, comp.f90:60-72), bound, then thermalconduction:
//   per axis the interface flux j = -kappa_eff (T_r - T_l) / d with
//   T = p / rho * temp0 (press2temp, comp.f90:87-102), and per cell
//   E += dt/d (j_l - j_r), S += (g-1) dE / rho^(g-1) (thermalintegration),
//   axes in the order x, y, z, every axis from the same primitives;
//   boundary cells from the same index map as the hydro update.
//
// kappa_eff = 1/(g-1) (simplekappa).  The time-step limit (thermalstep) is
// part of the CFL kernel.  This translation unit is compiled without FMA
// contraction.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "common.h"
#include "conduction.h"

namespace evora {
namespace {

constexpr int kThreads = 256;

int grid_of(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

// Boundary index map of one axis (boundary.f90:26-113); temperatures do not
// see the velocity reflection of boundary type 3.
__device__ __forceinline__ int map_ghost(int g, int n, int bt) {
  if (g >= 0 && g < n) return g;
  if (bt == 2) return g < 0 ? g + n : g - n;
  if (g < 0) return -g - 1;
  return 2 * n - g - 1;
}

// primitive(w,q) for the cells: the dual-energy resynchronisation written
// back to q, and T = p / rho * temp0 of every cell.
template <typename T>
__global__ void k_cond_prim(T* __restrict__ q, int64_t n, int nf, HydroParams P, double* __restrict__ temp,
                            const GridCtl* ctl, unsigned* err) {
  if (ctl_skip(ctl)) return;
  const Gas<double> c = Gas<double>::make(P);
  const bool de = P.dualenergy != 0;
  const double temp0 = units_of(P, ctl).temp0;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6], w[5];
    load_cell(q, n, nf, i, v);
    q2w(v, w, c, de, e);
    if (de) {
      q[4 * n + i] = (T)v[4];
      if (nf == 6) q[5 * n + i] = (T)v[5];
    }
    temp[i] = w[4] / w[0] * temp0;
  }
  if (e) atomicOr(err, e);
}

// thermalflux (conduction.f90:126-148), simplekappa branch.
__device__ __forceinline__ double thermal_flux(double tl, double tr, double deltainv, double g1) {
  const double kappa_eff = 1.0 / g1;
  const double dtempdx = (tr - tl) * deltainv;
  return -(kappa_eff * dtempdx);
}

template <typename T>
__global__ void k_cond_update(T* __restrict__ q, int64_t n, int nf, HydroParams P, const double* __restrict__ temp,
                              const GridCtl* ctl, double dt_host) {
  // 3D launch: x by threads, one (y, z) row per block row
  if (ctl_skip(ctl)) return;
  const double dt = ctl ? ctl->dt : dt_host;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int64_t nxy = (int64_t)nx * ny;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, iz = blockIdx.z;
  if (ix < nx) {
    const int64_t i = ((int64_t)iz * ny + iy) * nx + ix;
    const double tc = temp[i];
    double e = (double)q[4 * n + i];
    const bool carry_s = nf == 6;
    double s = carry_s ? (double)q[5 * n + i] : 0.0;
    // rho^(g-1) of the cell, the same in every axis's thermalintegration
    const double rg = carry_s ? pow((double)q[i], P.g1) : 1.0;
    auto integrate = [&](double tl, double tr, double deltainv) {
      const double jl = thermal_flux(tl, tc, deltainv, P.g1);
      const double jr = thermal_flux(tc, tr, deltainv, P.g1);
      const double delta = dt * deltainv;
      const double d = delta * (jl - jr);          // thermalintegration (150-164)
      e = e + d;
      if (carry_s) s = s + P.g1 * d / rg;
    };
    if (nx != 1) {
      const int64_t base = i - ix;
      integrate(temp[base + map_ghost(ix - 1, nx, P.boundtype)], temp[base + map_ghost(ix + 1, nx, P.boundtype)],
                P.dxinv);
    }
    if (ny != 1) {
      const int64_t base = i - (int64_t)iy * nx;
      integrate(temp[base + (int64_t)map_ghost(iy - 1, ny, P.boundtype) * nx],
                temp[base + (int64_t)map_ghost(iy + 1, ny, P.boundtype) * nx], P.dyinv);
    }
    if (nz != 1) {
      const int64_t base = i - (int64_t)iz * nxy;
      integrate(temp[base + (int64_t)map_ghost(iz - 1, nz, P.boundtype) * nxy],
                temp[base + (int64_t)map_ghost(iz + 1, nz, P.boundtype) * nxy], P.dzinv);
    }
    q[4 * n + i] = (T)e;
    if (nf == 6) q[5 * n + i] = (T)s;
  }
}

}  // namespace

int cond_plan(int64_t n, CondPlan* c) {
  cond_plan_free(c);
  c->n = n;
  if (cudaMalloc(&c->temp, sizeof(double) * n) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  return 0;
}

void cond_plan_free(CondPlan* c) {
  cudaFree(c->temp);
  *c = CondPlan{};
}

// ------------------------------------------------------------ drop-in --
namespace {

// Offset of w(1, ix, iy, iz) in w(5, -1:nx+2, -1:ny+2, -1:nz+2) (0-based
// interior indices; the ghost frame exists in every axis).
__device__ __forceinline__ int64_t w_at(const HydroParams& P, int ix, int iy, int iz) {
  return (int64_t)EVORA_NW * (((int64_t)(iz + 2) * (P.ny + 4) + (iy + 2)) * (P.nx + 4) + (ix + 2));
}

// thermalconduction(q, w) (conduction.f90:26-122) on the reference layouts:
// temperatures from w (ghosts included, as bound left them).
__global__ void k_cond_aos(double* __restrict__ q, const double* __restrict__ w, HydroParams P, double dt) {
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % P.nx);
    const int64_t r = i / P.nx;
    const int iy = (int)(r % P.ny), iz = (int)(r / P.ny);
    auto T = [&](int x, int y, int z) {
      const double* c = w + w_at(P, x, y, z);
      return c[4] / c[0] * P.temp0;
    };
    const double tc = T(ix, iy, iz);
    double* qc = q + (int64_t)EVORA_NQ * i;
    double e = qc[4], s = qc[5];
    const double rho = qc[0];
    auto integrate = [&](double tl, double tr, double deltainv) {
      const double jl = thermal_flux(tl, tc, deltainv, P.g1);
      const double jr = thermal_flux(tc, tr, deltainv, P.g1);
      const double d = (dt * deltainv) * (jl - jr);
      e = e + d;
      s = s + P.g1 * d / pow(rho, P.g1);
    };
    if (P.nx != 1) integrate(T(ix - 1, iy, iz), T(ix + 1, iy, iz), P.dxinv);
    if (P.ny != 1) integrate(T(ix, iy - 1, iz), T(ix, iy + 1, iz), P.dyinv);
    if (P.nz != 1) integrate(T(ix, iy, iz - 1), T(ix, iy, iz + 1), P.dzinv);
    qc[4] = e;
    qc[5] = s;
  }
}

// thermalstep (timestep.f90:72-104) part 1: min over cells of rho / kappa,
// rho from w and T from pressure(q) (which, with dual energy, also
// resynchronises q in place as the reference's call does).
__global__ void k_thermalstep_aos(double* __restrict__ q, const double* __restrict__ w, HydroParams P,
                                  unsigned long long* vmin_bits, unsigned* err) {
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const Gas<double> c = Gas<double>::make(P);
  double vmin = 1e99;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % P.nx);
    const int64_t r = i / P.nx;
    const int iy = (int)(r % P.ny), iz = (int)(r / P.ny);
    double* qc = q + (int64_t)EVORA_NQ * i;
    const double press = pressure(qc, c, P.dualenergy != 0, e);
    const double temp = press / qc[0] * P.temp0;
    const double kappa = P.kappa0 * pow(temp, 2.5);
    const double v = w[w_at(P, ix, iy, iz)] / kappa;
    if (v < vmin) vmin = v;
  }
  for (int off = 16; off > 0; off >>= 1) vmin = fmin2(vmin, __shfl_xor_sync(0xffffffffu, vmin, off));
  if ((threadIdx.x & 31) == 0) atomicMin(vmin_bits, ordered_bits(vmin));
  if (e) atomicOr(err, e);
}

struct DropinCond {
  std::mutex mu;
  int device = -1;
  double* q = nullptr;
  double* w = nullptr;
  size_t qbytes = 0, wbytes = 0;
  unsigned long long* scratch = nullptr;   // [0] vmin bits, [1] error word
};

DropinCond& dc() {
  static DropinCond s;
  return s;
}

int stage(double** buf, size_t* have, size_t need) {
  if (*have >= need) return 0;
  cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  if (cudaMalloc(buf, need) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  *have = need;
  return 0;
}

int finish(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_cuda_error(e, where);
    return EVORA_ERR_CUDA;
  }
  return 0;
}

// Resolves q and w (host arrays are staged, device arrays used in place).
int prepare(DropinCond& D, HydroParams* P, const double* q, const double* w, double** dq, double** dw) {
  if (!dropin_params(P)) return EVORA_ERR_ARG;
  if (!P->conduction || !P->simplekappa) return EVORA_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EVORA_ERR_CUDA;
  if (dev != D.device) {
    cudaFree(D.q);
    cudaFree(D.w);
    cudaFree(D.scratch);
    D.q = D.w = nullptr;
    D.scratch = nullptr;
    D.qbytes = D.wbytes = 0;
    D.device = dev;
  }
  if (!D.scratch && cudaMalloc(&D.scratch, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  const int64_t nq = (int64_t)EVORA_NQ * P->nx * P->ny * P->nz;
  const int64_t nw = (int64_t)EVORA_NW * (P->nx + 4) * (P->ny + 4) * (P->nz + 4);
  int rc;
  *dq = const_cast<double*>(q);
  *dw = const_cast<double*>(w);
  if (!is_device_pointer(q)) {
    if ((rc = stage(&D.q, &D.qbytes, nq * 8))) return rc;
    if (cudaMemcpy(D.q, q, nq * 8, cudaMemcpyHostToDevice) != cudaSuccess) return finish("conduction staging");
    *dq = D.q;
  }
  if (!is_device_pointer(w)) {
    if ((rc = stage(&D.w, &D.wbytes, nw * 8))) return rc;
    if (cudaMemcpy(D.w, w, nw * 8, cudaMemcpyHostToDevice) != cudaSuccess) return finish("conduction staging");
    *dw = D.w;
  }
  return 0;
}

}  // namespace

int cond_step(CondPlan& c, const HydroParams& P, void* q, bool f32, int nf, GridCtl* ctl, double dt_host,
              cudaStream_t st) {
  unsigned* err = &ctl->err;
  const dim3 rows((P.nx + 127) / 128, P.ny, P.nz);
  if (f32) {
    k_cond_prim<float><<<grid_of(c.n), kThreads, 0, st>>>((float*)q, c.n, nf, P, c.temp, ctl, err);
    k_cond_update<float><<<rows, 128, 0, st>>>((float*)q, c.n, nf, P, c.temp, ctl, dt_host);
  } else {
    k_cond_prim<double><<<grid_of(c.n), kThreads, 0, st>>>((double*)q, c.n, nf, P, c.temp, ctl, err);
    k_cond_update<double><<<rows, 128, 0, st>>>((double*)q, c.n, nf, P, c.temp, ctl, dt_host);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "thermalconduction");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

}  // namespace evora

using namespace evora;

extern "C" {

int evora_thermalstep(double* q, const double* w, double* dt) {
  if (!q || !w || !dt) return EVORA_ERR_ARG;
  evora::dropin_resident_read(q);
  DropinCond& D = dc();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  double *dq, *dw;
  int rc = prepare(D, &P, q, w, &dq, &dw);
  if (rc) return rc;
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const double big = 1e99;   // thermalstep's initial v (timestep.f90:82)
  unsigned long long init[2] = {0ull, 0ull};
  std::memcpy(&init[0], &big, sizeof big);
  if (cudaMemcpy(D.scratch, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess)
    return finish("evora_thermalstep");
  k_thermalstep_aos<<<grid_of(n), kThreads>>>(dq, dw, P, D.scratch, reinterpret_cast<unsigned*>(D.scratch + 1));
  if ((rc = finish("evora_thermalstep"))) return rc;
  unsigned long long out[2];
  if (cudaMemcpy(out, D.scratch, sizeof out, cudaMemcpyDeviceToHost) != cudaSuccess)
    return finish("evora_thermalstep");
  if (dq != q && cudaMemcpy(q, dq, sizeof(double) * EVORA_NQ * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return finish("evora_thermalstep");
  unsigned err = (unsigned)out[1];
  if (err) return (int)err;
  double vmin;
  std::memcpy(&vmin, &out[0], sizeof vmin);
  *dt = thermal_dt(P, units_of(P, nullptr), vmin, *dt, err);
  return (int)err;
}

int evora_thermalconduction(double* q, const double* w, double dt) {
  if (!q || !w) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinCond& D = dc();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  double *dq, *dw;
  int rc = prepare(D, &P, q, w, &dq, &dw);
  if (rc) return rc;
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  k_cond_aos<<<grid_of(n), kThreads>>>(dq, dw, P, dt);
  if ((rc = finish("evora_thermalconduction"))) return rc;
  if (dq != q && cudaMemcpy(q, dq, sizeof(double) * EVORA_NQ * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return finish("evora_thermalconduction");
  return 0;
}

}  // extern "C"
