// dropin_kernels.cuh -- kernels of the drop-in layer: one kernel (or a short
// sequence) per reference subroutine, working in place on the reference's
// own array layouts (column-major AoS, field index fastest, ghost frames of
// main.f90:72-75).  Included by dropin_fast.cu and dropin_strict.cu, which
// compile it with and without FMA contraction into namespaces `fast` and
// `strict`.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

#ifndef EVORA_NS
#error "define EVORA_NS before including dropin_kernels.cuh"
#endif

namespace evora {
namespace EVORA_NS {

// Reference array indexing, 1-based interior indices as in the Fortran.
// NQ, NW: the leading dimensions of q and of w, evo, s (global.f90:30-36:
// 6 and 5 in the plain build, 12 and 5 with -DCIE, 12 and 11 with -DNONCIE).
template <int NQ = EVORA_NQ, int NW = EVORA_NW>
struct RefLayout {
  int nx, ny, nz;
  __device__ __forceinline__ int64_t q(int i, int j, int k) const {   // q(nq, 1:nx, 1:ny, 1:nz)
    return (int64_t)NQ * ((int64_t)(i - 1) + (int64_t)nx * ((int64_t)(j - 1) + (int64_t)ny * (k - 1)));
  }
  __device__ __forceinline__ int64_t w(int i, int j, int k) const {   // w(nw, -1:nx+2, ...)
    return (int64_t)NW * ((int64_t)(i + 1) + (int64_t)(nx + 4) * ((int64_t)(j + 1) + (int64_t)(ny + 4) * (k + 1)));
  }
  __device__ __forceinline__ int64_t e(int i, int j, int k) const {   // evo(nw, 0:nx+1, ...)
    return (int64_t)NW * ((int64_t)i + (int64_t)(nx + 2) * ((int64_t)j + (int64_t)(ny + 2) * k));
  }
  __device__ __forceinline__ int64_t s(int d, int i, int j, int k) const {  // s(nw, 3, 0:nx+1, ...)
    return (int64_t)NW * ((int64_t)(d - 1) + 3 * ((int64_t)i + (int64_t)(nx + 2) * ((int64_t)j + (int64_t)(ny + 2) * k)));
  }
};

__device__ __forceinline__ void flush_err(unsigned* err, unsigned e) {
  if (e) atomicOr(err, e);
}

// primitive(w,q), muscl.f90:26-43: one thread per interior cell; with nw =
// 11 the species per unit mass w(6:11) = q(7:12) / rho (comp.f90:40-42).
template <int NQ, int NW>
__global__ void k_primitive(HydroParams P, double* __restrict__ w, double* __restrict__ q,
                            unsigned* err, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const RefLayout<NQ, NW> L{P.nx, P.ny, P.nz};
  const Gas<double> c = Gas<double>::make(P);
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  unsigned e = 0;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % P.nx) + 1;
    int j = (int)((idx / P.nx) % P.ny) + 1;
    int k = (int)(idx / ((int64_t)P.nx * P.ny)) + 1;
    double* qc = q + L.q(i, j, k);
    double qv[EVORA_NQ], wv[NW];
#pragma unroll
    for (int f = 0; f < EVORA_NQ; ++f) qv[f] = qc[f];
    q2w(qv, wv, c, P.dualenergy != 0, e);
    if (P.dualenergy) {
      qc[4] = qv[4];
      qc[5] = qv[5];
    }
    if (NW > 5) {
      const double densinv = 1.0 / qv[0];
#pragma unroll
      for (int f = 5; f < NW; ++f) wv[f] = qc[f + 1] * densinv;
    }
    double* wc = w + L.w(i, j, k);
#pragma unroll
    for (int f = 0; f < NW; ++f) wc[f] = wv[f];
  }
  flush_err(err, e);
}

// bound(w), boundary.f90:26-113.  One launch per axis, in the reference's
// order x, y, z, each over the full ghost-inclusive extent of the other two
// axes, so edges and corners end up as the reference leaves them.
template <int NW>
__device__ __forceinline__ void copy_cell(double* w, int64_t dst, int64_t src, bool reflect) {
  w[dst + 0] = w[src + 0];
  w[dst + 1] = reflect ? -w[src + 1] : w[src + 1];
  w[dst + 2] = reflect ? -w[src + 2] : w[src + 2];
  w[dst + 3] = reflect ? -w[src + 3] : w[src + 3];
#pragma unroll
  for (int f = 4; f < NW; ++f) w[dst + f] = w[src + f];
}

template <int NW>
__global__ void k_bound_x(HydroParams P, double* __restrict__ w, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const RefLayout<EVORA_NQ, NW> L{P.nx, P.ny, P.nz};
  const int ny4 = P.ny + 4, nz4 = P.nz + 4, nx = P.nx, bt = P.boundtype;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ny4 * nz4; idx += gridDim.x * blockDim.x) {
    int j = idx % ny4 - 1, k = idx / ny4 - 1;
    if (bt == 1 || bt == 3) {              // lower: zero gradient (41-48 unreachable)
      copy_cell<NW>(w, L.w(-1, j, k), L.w(2, j, k), false);
      copy_cell<NW>(w, L.w(0, j, k), L.w(1, j, k), false);
    } else if (bt == 2) {
      copy_cell<NW>(w, L.w(-1, j, k), L.w(nx - 1, j, k), false);
      copy_cell<NW>(w, L.w(0, j, k), L.w(nx, j, k), false);
    }
    if (bt == 1) {
      copy_cell<NW>(w, L.w(nx + 2, j, k), L.w(nx - 1, j, k), false);
      copy_cell<NW>(w, L.w(nx + 1, j, k), L.w(nx, j, k), false);
    } else if (bt == 2) {
      copy_cell<NW>(w, L.w(nx + 2, j, k), L.w(2, j, k), false);
      copy_cell<NW>(w, L.w(nx + 1, j, k), L.w(1, j, k), false);
    } else if (bt == 3) {                  // reflecting upper x face
      copy_cell<NW>(w, L.w(nx + 1, j, k), L.w(nx, j, k), true);
      copy_cell<NW>(w, L.w(nx + 2, j, k), L.w(nx - 1, j, k), true);
    }
  }
}

template <int NW>
__global__ void k_bound_y(HydroParams P, double* __restrict__ w, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const RefLayout<EVORA_NQ, NW> L{P.nx, P.ny, P.nz};
  const int nx4 = P.nx + 4, nz4 = P.nz + 4, ny = P.ny, bt = P.boundtype;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nx4 * nz4; idx += gridDim.x * blockDim.x) {
    int i = idx % nx4 - 1, k = idx / nx4 - 1;
    if (bt == 1 || bt == 3) {
      copy_cell<NW>(w, L.w(i, -1, k), L.w(i, 2, k), false);
      copy_cell<NW>(w, L.w(i, 0, k), L.w(i, 1, k), false);
      copy_cell<NW>(w, L.w(i, ny + 2, k), L.w(i, ny - 1, k), false);
      copy_cell<NW>(w, L.w(i, ny + 1, k), L.w(i, ny, k), false);
    } else if (bt == 2) {
      copy_cell<NW>(w, L.w(i, -1, k), L.w(i, ny - 1, k), false);
      copy_cell<NW>(w, L.w(i, 0, k), L.w(i, ny, k), false);
      copy_cell<NW>(w, L.w(i, ny + 2, k), L.w(i, 2, k), false);
      copy_cell<NW>(w, L.w(i, ny + 1, k), L.w(i, 1, k), false);
    }
  }
}

template <int NW>
__global__ void k_bound_z(HydroParams P, double* __restrict__ w, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const RefLayout<EVORA_NQ, NW> L{P.nx, P.ny, P.nz};
  const int nx4 = P.nx + 4, ny4 = P.ny + 4, nz = P.nz, bt = P.boundtype;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nx4 * ny4; idx += gridDim.x * blockDim.x) {
    int i = idx % nx4 - 1, j = idx / nx4 - 1;
    if (bt == 1 || bt == 3) {
      copy_cell<NW>(w, L.w(i, j, -1), L.w(i, j, 2), false);
      copy_cell<NW>(w, L.w(i, j, 0), L.w(i, j, 1), false);
      copy_cell<NW>(w, L.w(i, j, nz + 2), L.w(i, j, nz - 1), false);
      copy_cell<NW>(w, L.w(i, j, nz + 1), L.w(i, j, nz), false);
    } else if (bt == 2) {
      copy_cell<NW>(w, L.w(i, j, -1), L.w(i, j, nz - 1), false);
      copy_cell<NW>(w, L.w(i, j, 0), L.w(i, j, nz), false);
      copy_cell<NW>(w, L.w(i, j, nz + 2), L.w(i, j, 2), false);
      copy_cell<NW>(w, L.w(i, j, nz + 1), L.w(i, j, 1), false);
    }
  }
}

// hydrostep(w), timestep.f90:26-57, part 1: per-axis maxima of the signal
// speed |u_d| + a over the interior.  Because a correctly rounded division
// by a positive number is monotone, min over cells of dx/(|u|+a) equals
// dx/max(|u|+a) exactly, so the reduction keeps maxima and divides once.
// smax[0..2] hold the maxima as ordered u64 bit patterns (NaN speeds are
// skipped, as MIN skips them).
template <int NW>
__global__ void k_cfl(HydroParams P, const double* __restrict__ w, unsigned long long* smax,
                      const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  const RefLayout<EVORA_NQ, NW> L{P.nx, P.ny, P.nz};
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % P.nx) + 1;
    int j = (int)((idx / P.nx) % P.ny) + 1;
    int k = (int)(idx / ((int64_t)P.nx * P.ny)) + 1;
    const double* c = w + L.w(i, j, k);
    double a = sqrt(P.g * c[4] / c[0]);
    double s0 = fabs(c[1]) + a, s1 = fabs(c[2]) + a, s2 = fabs(c[3]) + a;
    if (s0 > m0) m0 = s0;
    if (s1 > m1) m1 = s1;
    if (s2 > m2) m2 = s2;
  }
  // warp then block reduction of the three maxima
  for (int off = 16; off > 0; off >>= 1) {
    m0 = fmax2(m0, __shfl_xor_sync(0xffffffffu, m0, off));
    m1 = fmax2(m1, __shfl_xor_sync(0xffffffffu, m1, off));
    m2 = fmax2(m2, __shfl_xor_sync(0xffffffffu, m2, off));
  }
  __shared__ double red[3][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0) { red[0][wid] = m0; red[1][wid] = m1; red[2][wid] = m2; }
  __syncthreads();
  if (wid == 0) {
    m0 = lane < nw ? red[0][lane] : 0.0;
    m1 = lane < nw ? red[1][lane] : 0.0;
    m2 = lane < nw ? red[2][lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) {
      m0 = fmax2(m0, __shfl_xor_sync(0xffffffffu, m0, off));
      m1 = fmax2(m1, __shfl_xor_sync(0xffffffffu, m1, off));
      m2 = fmax2(m2, __shfl_xor_sync(0xffffffffu, m2, off));
    }
    if (lane == 0) {
      atomicMax(&smax[0], ordered_bits(m0));
      atomicMax(&smax[1], ordered_bits(m1));
      atomicMax(&smax[2], ordered_bits(m2));
    }
  }
}

// compevo(w,evo,s), muscl.f90:45-113: one thread per cell of the interior
// plus one ghost layer (lx1:mx1 ...), with the 1D, 2D and 3D variants.
template <int NW>
__global__ void k_compevo(HydroParams P, const double* __restrict__ w, double* __restrict__ evo,
                          double* __restrict__ s, double dt, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  if (ctl) dt = ctl->dt;
  const RefLayout<EVORA_NQ, NW> L{P.nx, P.ny, P.nz};
  const double dt2 = -0.5 * dt;
  const int ex = P.nx + 2;
  const int ey = P.onedimension ? 1 : P.ny + 2;
  const int ez = P.twodimension ? 1 : P.nz + 2;
  const int64_t n = (int64_t)ex * ey * ez;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % ex);
    int j = (int)((idx / ex) % ey);
    int k = (int)(idx / ((int64_t)ex * ey));
    if (P.onedimension) j = 1;
    if (P.twodimension) k = 1;
    const double* wc = w + L.w(i, j, k);
    double wv[NW];
#pragma unroll
    for (int f = 0; f < NW; ++f) wv[f] = wc[f];
    const int ndim = P.onedimension ? 1 : (P.twodimension ? 2 : 3);
    double a[3][NW];
    for (int d = 1; d <= ndim; ++d) {
      const double* wm = w + (d == 1 ? L.w(i - 1, j, k) : d == 2 ? L.w(i, j - 1, k) : L.w(i, j, k - 1));
      const double* wp = w + (d == 1 ? L.w(i + 1, j, k) : d == 2 ? L.w(i, j + 1, k) : L.w(i, j, k + 1));
      double sv[NW];
#pragma unroll
      for (int f = 0; f < NW; ++f) sv[f] = slope1(wm[f], wv[f], wp[f], P.limiter);
      double* sd = s + L.s(d, i, j, k);
#pragma unroll
      for (int f = 0; f < NW; ++f) sd[f] = sv[f];
      predictor_term(wv, sv, d, P.g, a[d - 1]);
      // species rows: the advection term alone (muscl.f90:62, 73-74, 92-94)
#pragma unroll
      for (int f = 5; f < NW; ++f) a[d - 1][f] = wv[d] * sv[f];
    }
    double* e = evo + L.e(i, j, k);
    if (ndim == 1) {
#pragma unroll
      for (int f = 0; f < NW; ++f) e[f] = dt2 * a[0][f] * P.dxinv;           // 68
    } else if (ndim == 2) {
#pragma unroll
      for (int f = 0; f < NW; ++f) e[f] = dt2 * (a[0][f] * P.dxinv + a[1][f] * P.dyinv);  // 86
    } else {
#pragma unroll
      for (int f = 0; f < NW; ++f)
        e[f] = dt2 * (a[0][f] * P.dxinv + a[1][f] * P.dyinv + a[2][f] * P.dzinv);  // 106-107
    }
  }
}

// sweep(w,q,evo,s), muscl.f90:171-274: one thread per interior cell.  The
// flux through each face is a pure function of the two face states, so the
// cell computes the fluxes through its lower and upper faces itself (the
// reference reuses fr as the next cell's fl; the values are identical).
// The x, y, z contributions are added in that order (integration,
// muscl.f90:276-290).
template <int NQ, int NW, int NF>
__global__ void k_sweep(HydroParams P, const double* __restrict__ w, double* __restrict__ q,
                        const double* __restrict__ evo, const double* __restrict__ s, double dt,
                        unsigned* err, const GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  if (ctl) dt = ctl->dt;
  const RefLayout<NQ, NW> L{P.nx, P.ny, P.nz};
  const Gas<double> c = Gas<double>::make(P);
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  const bool so = P.secondorder != 0;
  unsigned e = 0;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(idx % P.nx) + 1;
    int j = (int)((idx / P.nx) % P.ny) + 1;
    int k = (int)(idx / ((int64_t)P.nx * P.ny)) + 1;
    double qv[NF];
    double* qc = q + L.q(i, j, k);
#pragma unroll
    for (int f = 0; f < NF; ++f) qv[f] = qc[f];
    for (int d = 1; d <= 3; ++d) {
      const int nd = d == 1 ? P.nx : d == 2 ? P.ny : P.nz;
      if (nd == 1) continue;
      const double delta = dt * (d == 1 ? P.dxinv : d == 2 ? P.dyinv : P.dzinv);
      const int di = d == 1, dj = d == 2, dk = d == 3;
      double fl[NF], fr[NF];
      for (int side = 0; side < 2; ++side) {
        // interface between cells a = (i,j,k) - 1 + side and b = a + 1 along d
        const int ai = i - di + side * di, aj = j - dj + side * dj, ak = k - dk + side * dk;
        const int bi = ai + di, bj = aj + dj, bk = ak + dk;
        const double* wa = w + L.w(ai, aj, ak);
        const double* wb = w + L.w(bi, bj, bk);
        double wl[NW], wr[NW];
        if (so) {
          const double* sa = s + L.s(d, ai, aj, ak);
          const double* sb = s + L.s(d, bi, bj, bk);
          const double* ea = evo + L.e(ai, aj, ak);
          const double* eb = evo + L.e(bi, bj, bk);
#pragma unroll
          for (int f = 0; f < NW; ++f) {
            wl[f] = face_plus(wa[f], sa[f], ea[f]);
            wr[f] = face_minus(wb[f], sb[f], eb[f]);
          }
        } else {
#pragma unroll
          for (int f = 0; f < NW; ++f) { wl[f] = wa[f]; wr[f] = wb[f]; }
        }
        riemann<double, NF>(wl, wr, side == 0 ? fl : fr, d, P.solver, c, e);
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) qv[f] = qv[f] + delta * (fl[f] - fr[f]);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) qc[f] = qv[f];
  }
  flush_err(err, e);
}

// Launchers (host).  Grid-stride kernels: grids sized to the SM count.
inline int grid_for(int64_t n, int block) {
  int64_t g = (n + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

template <int NQ, int NW>
inline void launch_primitive(const HydroParams& P, double* w, double* q, unsigned* err,
                             const GridCtl* ctl, cudaStream_t st) {
  int64_t n = (int64_t)P.nx * P.ny * P.nz;
  k_primitive<NQ, NW><<<grid_for(n, 256), 256, 0, st>>>(P, w, q, err, ctl);
}

template <int NW>
inline void launch_bound(const HydroParams& P, double* w, const GridCtl* ctl, cudaStream_t st) {
  if (P.nx != 1) k_bound_x<NW><<<grid_for((int64_t)(P.ny + 4) * (P.nz + 4), 256), 256, 0, st>>>(P, w, ctl);
  if (P.ny != 1) k_bound_y<NW><<<grid_for((int64_t)(P.nx + 4) * (P.nz + 4), 256), 256, 0, st>>>(P, w, ctl);
  if (P.nz != 1) k_bound_z<NW><<<grid_for((int64_t)(P.nx + 4) * (P.ny + 4), 256), 256, 0, st>>>(P, w, ctl);
}

template <int NW>
inline void launch_cfl(const HydroParams& P, const double* w, unsigned long long* smax,
                       const GridCtl* ctl, cudaStream_t st) {
  int64_t n = (int64_t)P.nx * P.ny * P.nz;
  k_cfl<NW><<<grid_for(n, 256), 256, 0, st>>>(P, w, smax, ctl);
}

template <int NW>
inline void launch_compevo(const HydroParams& P, const double* w, double* evo, double* s, double dt,
                           const GridCtl* ctl, cudaStream_t st) {
  int64_t n = (int64_t)(P.nx + 2) * (P.onedimension ? 1 : P.ny + 2) * (P.twodimension ? 1 : P.nz + 2);
  k_compevo<NW><<<grid_for(n, 128), 128, 0, st>>>(P, w, evo, s, dt, ctl);
}

template <int NQ, int NW, int NF>
inline void launch_sweep(const HydroParams& P, const double* w, double* q, const double* evo,
                         const double* s, double dt, unsigned* err, const GridCtl* ctl, cudaStream_t st) {
  int64_t n = (int64_t)P.nx * P.ny * P.nz;
  k_sweep<NQ, NW, NF><<<grid_for(n, 128), 128, 0, st>>>(P, w, q, evo, s, dt, err, ctl);
}

}  // namespace EVORA_NS
}  // namespace evora
