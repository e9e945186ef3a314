// gravity.cu -- self-gravity on the device, the reference's
// gravitation.f90:
//
//   gravpotential  source grav (rho - <rho>), or a grav (rho / fb - 1) with
//                  comoving coordinates, forward FFT, multigreen (the
//                  discrete Green's function -h2 / sum_d sin^2(k_d pi / n_d)
//                  over n3), backward FFT                (26-53, 55-84)
//   gravintegration  centred potential differences (grav_force, periodic)
//                  and the source terms of E and m       (170-243)
//
// The reference transforms the real source as complex data (FFTW 2
// C2C); here the transforms are cuFFT D2Z / Z2D over the half spectrum,
// which gives the same potential up to rounding (FFTW 2.1.5 is not part of
// the reference tree, so this part has no bit-level reference; it is
// checked against a restatement with numpy's FFT and against the discrete
// Laplacian it inverts).  This translation unit is compiled without FMA
// contraction.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/evora_gpu.h"
#include "common.h"
#include "cosmology.cuh"
#include "gravity.h"

namespace evora {
namespace {

constexpr int kThreads = 256;
constexpr int kRow = 128;   // threads along x of the row-mapped (3D) launches

int grid_of(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

template <typename T>
__device__ __forceinline__ double rho_of(const T* q, int64_t n, int aos, int64_t i) {
  return aos ? (double)q[6 * i] : (double)q[i];
}

// sum(q(1, :, :, :)) in a fixed order: per-block partial sums, then one
// block over the partials; mean = sum / n3 (gravitation.f90:40-43).
template <typename T>
__global__ void k_rho_partial(const T* __restrict__ q, int64_t n, int aos, double* part, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += rho_of(q, n, aos, i);
  __shared__ double red[kThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// one block of kThreads: strided partial sums, then a fixed tree
__global__ void k_rho_mean(double* part, int nb, int64_t n, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  __shared__ double red[kThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += kThreads) s += part[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[nb] = red[0] / (double)n;
}

template <typename T>
__global__ void k_source(const T* __restrict__ q, int64_t n, int aos, const double* mean, double grav,
                         double* __restrict__ phi, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const double m = *mean;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    phi[i] = grav * (rho_of(q, n, aos, i) - m);
}

// The comoving source cosmo * grav * (rho / fb - 1) with grav = 1.5 omega0
// (gravitation.f90:36-37); cosmo from the grid's control block, or
// cosmo_host without one.
template <typename T>
__global__ void k_source_comoving(const T* __restrict__ q, int64_t n, int aos, double grav, double fb,
                                  double cosmo_host, double* __restrict__ phi, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const double cg = (ctl ? ctl->cosmo : cosmo_host) * grav;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    phi[i] = cg * (rho_of(q, n, aos, i) / fb - 1.0);
}

// multigreen (gravitation.f90:55-84) on the half spectrum (x index 0..nx/2):
// phi_k = phi_k / n3 * green, green = -h2 / (sin2x + sin2y + sin2z), 0 for k = 0.
__global__ void k_green(cufftDoubleComplex* __restrict__ spec, int nxh, int ny, int nz, const double* __restrict__ sx,
                        const double* __restrict__ sy, const double* __restrict__ sz, double h2, int64_t n3,
                        const GridCtl* ctl) {
  // 3D launch: x by threads, one (y, z) row per block row
  if (ctl_skip(ctl)) return;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, iz = blockIdx.z;
  if (ix >= nxh) return;
  const double dn3 = (double)n3;
  const int64_t j = ((int64_t)iz * ny + iy) * nxh + ix;
  const double green = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : -h2 / (sx[ix] + sy[iy] + sz[iz]);
  cufftDoubleComplex v = spec[j];
  v.x = v.x / dn3 * green;
  v.y = v.y / dn3 * green;
  spec[j] = v;
}

// gravintegration + grav_force (gravitation.f90:170-243): periodic centred
// differences of phi; E gains dt (m . f) with the momentum before its
// update, then m gains dt rho f.  With EXPAND (a comoving step whose next
// substep is expansion(q), cosmology.f90:53-72, with nothing in between)
// the cell's expansion terms follow in the same pass: pressure() of the
// updated cell, E -= dt g35 expand p / g1, S -= dt g35 expand S -- the same
// per-cell arithmetic as the separate pass, without its trip through HBM.
template <typename T, bool EXPAND>
__global__ void k_integrate(T* __restrict__ q, int64_t n, int nf, int aos, const double* __restrict__ phi, int nx,
                            int ny, int nz, double dx2inv, double dy2inv, double dz2inv, const GridCtl* ctl,
                            double dt_host, HydroParams P) {
  // (the entropy field, when carried, is not touched by gravintegration:
  // it updates E and m only)
  // 3D launch: x by threads, one (y, z) row per block row
  if (ctl_skip(ctl)) return;
  const double dt = ctl ? ctl->dt : dt_host;
  const int64_t nxy = (int64_t)nx * ny;
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, iz = blockIdx.z;
  if (ix < nx) {
    const int64_t i = ((int64_t)iz * ny + iy) * nx + ix;
    double f1 = 0.0, f2 = 0.0, f3 = 0.0;
    if (nx != 1) {
      const int xp = ix + 1 == nx ? 0 : ix + 1, xm = ix == 0 ? nx - 1 : ix - 1;
      f1 = -(phi[i - ix + xp] - phi[i - ix + xm]) * dx2inv;
    }
    if (ny != 1) {
      const int yp = iy + 1 == ny ? 0 : iy + 1, ym = iy == 0 ? ny - 1 : iy - 1;
      f2 = -(phi[i + (int64_t)(yp - iy) * nx] - phi[i + (int64_t)(ym - iy) * nx]) * dy2inv;
    }
    if (nz != 1) {
      const int zp = iz + 1 == nz ? 0 : iz + 1, zm = iz == 0 ? nz - 1 : iz - 1;
      f3 = -(phi[i + (int64_t)(zp - iz) * nxy] - phi[i + (int64_t)(zm - iz) * nxy]) * dz2inv;
    }
    double v[6];
#pragma unroll
    for (int f = 0; f < 5; ++f) v[f] = aos ? (double)q[6 * i + f] : (double)q[f * n + i];
    v[4] = v[4] + dt * (v[1] * f1 + v[2] * f2 + v[3] * f3);
    v[1] = v[1] + dt * v[0] * f1;
    v[2] = v[2] + dt * v[0] * f2;
    v[3] = v[3] + dt * v[0] * f3;
    if (EXPAND) {
      // grid states only (aos = 0); S is 0 when not carried
      v[5] = nf == 6 ? (double)q[5 * n + i] : 0.0;
      unsigned err = 0;
      const double press = pressure(v, Gas<double>::make(P), P.dualenergy != 0, err);
      const double k = dt * P.g35 * ctl->expand;
      v[4] = v[4] - k * press / P.g1;
      v[5] = v[5] - k * v[5];
      if (nf == 6) q[5 * n + i] = (T)v[5];
      if (err) atomicOr(const_cast<unsigned*>(&ctl->err), err);
    }
#pragma unroll
    for (int f = 1; f < 5; ++f) {
      if (aos) q[6 * i + f] = (T)v[f];
      else q[f * n + i] = (T)v[f];
    }
  }
}

}  // namespace

int grav_plan(const HydroParams& P, GravPlan* g, cudaStream_t st) {
  grav_plan_free(g);
  g->nx = P.nx;
  g->ny = P.ny;
  g->nz = P.nz;
  g->n = (int64_t)P.nx * P.ny * P.nz;
  const int nxh = P.nx / 2 + 1;
  g->nh = (int64_t)nxh * P.ny * P.nz;
  // grav (parameter.f90:236-241): 1.5 omega0 with supercomoving, else
  // fourpig (global.f90:101)
  g->comoving = P.supercomoving != 0;
  g->grav = g->comoving ? P.gravc : 8.38553911e-7;
  g->fb = P.fb;
  g->dx2inv = 0.5 / P.dx;             // parameter.f90:219
  g->dy2inv = 0.5 / P.dy;
  g->dz2inv = 0.5 / P.dz;
  g->h2 = P.dx * P.dx / 4.0;          // dx ** 2.0 / 4.0 (parameter.f90:254)
  g->stream = st;
  // sin^2 tables (parameter.f90:255-263, comp.f90:241-252): kf = 2 pi / n
  // with module global's pi = (double)3.1415927f, the argument kf/2 * k
  const double pi = (double)3.1415927f;
  auto table = [&](int n, int count, std::vector<double>& out) {
    const int nyq = std::max(n / 2, 1);
    const double kf = 2.0 * pi / n, kf2 = kf * 0.5;
    for (int c = 0; c < count; ++c) {
      const int i = c + 1;
      const double k = i <= nyq ? (double)(i - 1) : -(double)(n - (i - 1));
      const double s = std::sin(kf2 * k);
      out.push_back(s * s);
    }
  };
  std::vector<double> tab;
  table(P.nx, nxh, tab);
  table(P.ny, P.ny, tab);
  table(P.nz, P.nz, tab);
  const int64_t b = (g->n + kThreads - 1) / kThreads;
  g->nred = (int)(b > 148 * 4 ? 148 * 4 : b);
  size_t bytes_phi = sizeof(double) * g->n, bytes_spec = sizeof(cufftDoubleComplex) * g->nh;
  if (cudaMalloc(&g->phi, bytes_phi) != cudaSuccess || cudaMalloc(&g->spec, bytes_spec) != cudaSuccess ||
      cudaMalloc(&g->green, sizeof(double) * tab.size()) != cudaSuccess ||
      cudaMalloc(&g->red, sizeof(double) * (g->nred + 1)) != cudaSuccess) {
    cudaGetLastError();
    grav_plan_free(g);
    return EVORA_ERR_NOMEM;
  }
  if (cudaMemcpy(g->green, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    grav_plan_free(g);
    return EVORA_ERR_CUDA;
  }
  // rank = number of axes longer than one (cuFFT plans want sizes >= 2)
  int dims[3], rank = 0;
  if (P.nz > 1) dims[rank++] = P.nz;
  if (P.ny > 1) dims[rank++] = P.ny;
  dims[rank++] = P.nx;
  if (cufftPlanMany(&g->fwd, rank, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1) != CUFFT_SUCCESS ||
      cufftPlanMany(&g->inv, rank, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 1) != CUFFT_SUCCESS) {
    set_error_message("cufftPlanMany failed");
    grav_plan_free(g);
    return EVORA_ERR_CUDA;
  }
  grav_set_stream(g, st);
  g->ready = true;
  return 0;
}

void grav_set_stream(GravPlan* g, cudaStream_t st) {
  g->stream = st;
  if (g->fwd) cufftSetStream(g->fwd, st);
  if (g->inv) cufftSetStream(g->inv, st);
}

void grav_plan_free(GravPlan* g) {
  if (g->fwd) cufftDestroy(g->fwd);
  if (g->inv) cufftDestroy(g->inv);
  cudaFree(g->phi);
  cudaFree(g->spec);
  cudaFree(g->green);
  cudaFree(g->red);
  *g = GravPlan{};
}

int grav_potential(GravPlan& g, const void* q, bool f32, int nf, int aos, const GridCtl* ctl, double cosmo_host) {
  (void)nf;
  cudaStream_t st = g.stream;
  if (g.comoving) {
    if (f32)
      k_source_comoving<float><<<grid_of(g.n), kThreads, 0, st>>>((const float*)q, g.n, aos, g.grav, g.fb, cosmo_host,
                                                                   g.phi, ctl);
    else
      k_source_comoving<double><<<grid_of(g.n), kThreads, 0, st>>>((const double*)q, g.n, aos, g.grav, g.fb,
                                                                    cosmo_host, g.phi, ctl);
  } else {
    if (f32) {
      k_rho_partial<float><<<g.nred, kThreads, 0, st>>>((const float*)q, g.n, aos, g.red, ctl);
    } else {
      k_rho_partial<double><<<g.nred, kThreads, 0, st>>>((const double*)q, g.n, aos, g.red, ctl);
    }
    k_rho_mean<<<1, kThreads, 0, st>>>(g.red, g.nred, g.n, ctl);   // the tree needs all kThreads threads
    if (f32) {
      k_source<float><<<grid_of(g.n), kThreads, 0, st>>>((const float*)q, g.n, aos, g.red + g.nred, g.grav, g.phi,
                                                          ctl);
    } else {
      k_source<double><<<grid_of(g.n), kThreads, 0, st>>>((const double*)q, g.n, aos, g.red + g.nred, g.grav, g.phi,
                                                          ctl);
    }
  }
  if (cufftExecD2Z(g.fwd, g.phi, g.spec) != CUFFT_SUCCESS) {
    set_error_message("cufftExecD2Z failed");
    return EVORA_ERR_CUDA;
  }
  const int nxh = g.nx / 2 + 1;
  const dim3 gh((nxh + kRow - 1) / kRow, g.ny, g.nz);
  k_green<<<gh, kRow, 0, st>>>(g.spec, nxh, g.ny, g.nz, g.green, g.green + nxh, g.green + nxh + g.ny, g.h2, g.n,
                               ctl);
  if (cufftExecZ2D(g.inv, g.spec, g.phi) != CUFFT_SUCCESS) {
    set_error_message("cufftExecZ2D failed");
    return EVORA_ERR_CUDA;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "gravpotential");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

int grav_integrate(GravPlan& g, void* q, bool f32, int nf, int aos, const GridCtl* ctl, double dt_host,
                   const HydroParams* expand) {
  cudaStream_t st = g.stream;
  const dim3 rows((g.nx + kRow - 1) / kRow, g.ny, g.nz);
  if (expand && (aos || !ctl)) return EVORA_ERR_ARG;   // the fused expansion reads dt, expand from a grid
  const HydroParams P = expand ? *expand : HydroParams{};
  if (f32) {
    auto k = expand ? k_integrate<float, true> : k_integrate<float, false>;
    k<<<rows, kRow, 0, st>>>((float*)q, g.n, nf, aos, g.phi, g.nx, g.ny, g.nz, g.dx2inv, g.dy2inv, g.dz2inv, ctl,
                             dt_host, P);
  } else {
    auto k = expand ? k_integrate<double, true> : k_integrate<double, false>;
    k<<<rows, kRow, 0, st>>>((double*)q, g.n, nf, aos, g.phi, g.nx, g.ny, g.nz, g.dx2inv, g.dy2inv, g.dz2inv, ctl,
                             dt_host, P);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e, "gravintegration");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

// ------------------------------------------------------------ drop-in --
namespace {

__global__ void k_real_to_complex(const double* __restrict__ re, double* __restrict__ c, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    c[2 * i] = re[i];
    c[2 * i + 1] = 0.0;
  }
}

__global__ void k_complex_to_real(const double* __restrict__ c, double* __restrict__ re, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    re[i] = c[2 * i];
}

// The drop-in layer's solve: one plan for the module-global grid, staging
// buffers for host arrays.
struct DropinGrav {
  std::mutex mu;
  GravPlan plan;
  int device = -1;
  double* q = nullptr;
  double* phi = nullptr;   // complex(8) phi(n3), interleaved
  int64_t n = 0;
};

DropinGrav& dg() {
  static DropinGrav s;
  return s;
}

int dropin_prepare(DropinGrav& D, HydroParams* P) {
  if (!dropin_params(P)) return EVORA_ERR_ARG;
  if (P->chemistry) return EVORA_ERR_ARG;   // the drop-in reads q(6, ...); grids take q(12, ...)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EVORA_ERR_CUDA;
  const int64_t n = (int64_t)P->nx * P->ny * P->nz;
  if (D.plan.ready && D.device == dev && D.plan.nx == P->nx && D.plan.ny == P->ny && D.plan.nz == P->nz &&
      D.plan.dx2inv == 0.5 / P->dx && D.plan.dy2inv == 0.5 / P->dy && D.plan.dz2inv == 0.5 / P->dz)
    return 0;
  grav_plan_free(&D.plan);
  cudaFree(D.q);
  cudaFree(D.phi);
  D.q = D.phi = nullptr;
  D.device = dev;
  D.n = n;
  int rc = grav_plan(*P, &D.plan, nullptr);
  if (rc) return rc;
  if (cudaMalloc(&D.q, sizeof(double) * EVORA_NQ * n) != cudaSuccess ||
      cudaMalloc(&D.phi, sizeof(double) * 2 * n) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  return 0;
}

int sync_status(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_cuda_error(e, where);
    return EVORA_ERR_CUDA;
  }
  return 0;
}

}  // namespace
}  // namespace evora

using namespace evora;

extern "C" {

int evora_gravpotential(const double* q, double* phi) {
  if (!q || !phi) return EVORA_ERR_ARG;
  evora::dropin_resident_read(q);
  DropinGrav& D = dg();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  int rc = dropin_prepare(D, &P);
  if (rc) return rc;
  const bool qdev = is_device_pointer(q), pdev = is_device_pointer(phi);
  const double* dq = q;
  if (!qdev) {
    if (cudaMemcpy(D.q, q, sizeof(double) * EVORA_NQ * D.n, cudaMemcpyHostToDevice) != cudaSuccess)
      return sync_status("evora_gravpotential");
    dq = D.q;
  }
  // the source of the current parameters, a from evora_settime
  D.plan.comoving = P.supercomoving != 0;
  D.plan.grav = D.plan.comoving ? P.gravc : 8.38553911e-7;
  D.plan.fb = P.fb;
  CosmoTime s;
  if (!dropin_time(&s)) return EVORA_ERR_ARG;
  if ((rc = grav_potential(D.plan, dq, false, EVORA_NQ, 1, nullptr, s.cosmo))) return rc;
  double* out = pdev ? phi : D.phi;
  k_real_to_complex<<<grid_of(D.n), kThreads>>>(D.plan.phi, out, D.n);
  if (!pdev && cudaMemcpy(phi, D.phi, sizeof(double) * 2 * D.n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return sync_status("evora_gravpotential");
  return sync_status("evora_gravpotential");
}

int evora_gravintegration(double* q, const double* phi, double dt) {
  if (!q || !phi) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinGrav& D = dg();
  std::lock_guard<std::mutex> lk(D.mu);
  HydroParams P;
  int rc = dropin_prepare(D, &P);
  if (rc) return rc;
  const bool qdev = is_device_pointer(q), pdev = is_device_pointer(phi);
  double* dq = q;
  if (!qdev) {
    if (cudaMemcpy(D.q, q, sizeof(double) * EVORA_NQ * D.n, cudaMemcpyHostToDevice) != cudaSuccess)
      return sync_status("evora_gravintegration");
    dq = D.q;
  }
  const double* dphi = phi;
  if (!pdev) {
    if (cudaMemcpy(D.phi, phi, sizeof(double) * 2 * D.n, cudaMemcpyHostToDevice) != cudaSuccess)
      return sync_status("evora_gravintegration");
    dphi = D.phi;
  }
  k_complex_to_real<<<grid_of(D.n), kThreads>>>(dphi, D.plan.phi, D.n);
  if ((rc = grav_integrate(D.plan, dq, false, EVORA_NQ, 1, nullptr, dt))) return rc;
  if (!qdev && cudaMemcpy(q, D.q, sizeof(double) * EVORA_NQ * D.n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return sync_status("evora_gravintegration");
  return sync_status("evora_gravintegration");
}

}  // extern "C"
