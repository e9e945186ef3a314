// fused.cu -- planning, layout conversion and diagnostics of the fused
// (structure-of-arrays) backend.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>

#include "../../include/evora_gpu.h"
#include "common.h"
#include "fused.h"

namespace evora {

namespace {
struct Inst {
  FusedLaunch (*pick)(int, int, int, int*, int*, int*, size_t*, int*, int*);
  int (*tiles)();
  void (*cfl)(const FusedPlan&, const void*, GridCtl*, cudaStream_t);
  bool (*fits)(const HydroParams&, int, int, int);
};
Inst inst_of(int precision, int strict) {
  if (precision == EVORA_FP32) return {f32::pick, f32::tiles, f32::cfl, f32::tile_fits};
  if (strict) return {f64s::pick, f64s::tiles, f64s::cfl, f64s::tile_fits};
  return {f64::pick, f64::tiles, f64::cfl, f64::tile_fits};
}
}  // namespace

// Planes per CTA of the 3D march.  The grid has tiles_xy x chunks CTAs, run
// in waves of SMs x CTAs-per-SM; the last wave is partly empty, and every
// chunk reloads two planes of halo.  The choice maximises
// (waves / ceil(waves)) x zc / (zc + 2) over chunk counts with zc >= 16
// (EVORA_ZC overrides).
int choose_zc(const HydroParams& P, int tx, int ty, int minb, int zc_default) {
  if (const char* e = getenv("EVORA_ZC")) {
    const int z = atoi(e);
    if (z > 0) return z;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  const long long tiles_xy = (long long)((P.nx + tx - 1) / tx) * ((P.ny + ty - 1) / ty);
  const double slots = (double)sms * (minb > 0 ? minb : 1);
  double best = -1.0;
  int best_zc = zc_default;
  for (int chunks = 1; chunks <= P.nz; ++chunks) {
    const int zc = (P.nz + chunks - 1) / chunks;
    if (zc < 16 && chunks > 1) break;
    if ((P.nz + zc - 1) / zc != chunks) continue;   // the same split as a smaller count
    const double waves = (double)(tiles_xy * chunks) / slots;
    const double score = waves / std::ceil(waves) * (double)zc / (zc + 2);
    if (score > best + 1e-9) {
      best = score;
      best_zc = zc;
    }
  }
  return best_zc;
}

void fused_set_tile(FusedPlan* pl, int tile) {
  const Inst in = inst_of(pl->precision, pl->strict);
  if (tile < 0 || tile >= in.tiles()) tile = 0;
  if (!in.fits(pl->P, pl->nf, pl->dim, tile)) tile = 0;
  pl->tile = tile;
  pl->launch = in.pick(pl->nf, pl->dim, tile, &pl->tx, &pl->ty, &pl->zc, &pl->smem, &pl->threads, &pl->minb);
  const HydroParams& P = pl->P;
  if (pl->dim == 3) pl->zc = choose_zc(P, pl->tx, pl->ty, pl->minb, pl->zc);
  if (pl->dim == 1) {
    int64_t b = (P.nx + 127) / 128;
    pl->grid = dim3((unsigned)(b < 1 ? 1 : b), 1, 1);
  } else {
    pl->grid = dim3((P.nx + pl->tx - 1) / pl->tx, (P.ny + pl->ty - 1) / pl->ty,
                    pl->dim == 3 ? (P.nz + pl->zc - 1) / pl->zc : 1);
  }
}

int fused_tiles(const FusedPlan& pl) { return inst_of(pl.precision, pl.strict).tiles(); }

int fused_plan(const HydroParams& P, int precision, int nf, int strict, FusedPlan* pl, cudaStream_t astream) {
  *pl = FusedPlan{};
  pl->P = P;
  pl->precision = precision;
  pl->nf = nf;
  pl->strict = strict;
  pl->dim = P.onedimension ? 1 : (P.twodimension ? 2 : 3);
  pl->n = (int64_t)P.nx * P.ny * P.nz;
  if ((int64_t)P.nx * P.ny * P.nz >= ((int64_t)1 << 31)) return EVORA_ERR_ARG;  // in-field index is 32-bit
  pl->cfl = inst_of(precision, strict).cfl;
  pl->cfl_fused = pl->dim >= 2 ? 1 : 0;
  int tile = 0;
  if (const char* e = getenv("EVORA_TILE")) tile = atoi(e);
  fused_set_tile(pl, tile);
  int64_t nb = (pl->n + 255) / 256;
  pl->nblk_tot = (int)(nb > 148 * 4 ? 148 * 4 : nb);
  pl->alloc_stream = astream;
  const size_t pbytes = sizeof(double) * 6 * (pl->nblk_tot + 1);
  const cudaError_t ae = astream ? cudaMallocAsync((void**)&pl->partials, pbytes, astream)
                                 : cudaMalloc(&pl->partials, pbytes);
  if (ae != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  return 0;
}

void fused_plan_free(FusedPlan* pl) {
  if (pl->partials) {
    if (pl->alloc_stream) cudaFreeAsync(pl->partials, pl->alloc_stream);
    else cudaFree(pl->partials);
  }
  pl->partials = nullptr;
}

void fused_cfl(const FusedPlan& pl, const void* q, GridCtl* ctl, cudaStream_t st) { pl.cfl(pl, q, ctl, st); }

MultiLaunch fused_multi_pick(int precision, int strict, int nf, int* tx, int* ty, int* zc, size_t* smem,
                             int* threads, int* ctas_per_sm) {
  if (precision == EVORA_FP32) return f32::multi_pick(nf, tx, ty, zc, smem, threads, ctas_per_sm);
  if (strict) return f64s::multi_pick(nf, tx, ty, zc, smem, threads, ctas_per_sm);
  return f64::multi_pick(nf, tx, ty, zc, smem, threads, ctas_per_sm);
}

void fused_update(const FusedPlan& pl, const void* qin, void* qout, GridCtl* ctl, cudaStream_t st) {
  pl.launch(pl, qin, qout, ctl, st);
}

namespace {

// q(nq, cell) -> SoA state; with the chemistry build (nq = 12) the species
// q(7:12) go to their own FP64 field-major array.
template <typename T>
__global__ void k_from_aos(const double* __restrict__ aos, T* __restrict__ q, int64_t n, int nf, int nq,
                           double* __restrict__ species) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int f = 0; f < nf; ++f) q[f * n + i] = (T)aos[(int64_t)nq * i + f];
    if (species)
      for (int s = 0; s < nq - EVORA_NQ; ++s) species[s * n + i] = aos[(int64_t)nq * i + EVORA_NQ + s];
  }
}

// Without the entropy field, q(6) = p / rho^(g-1) of the current state
// (the value pressure() would resynchronise it to, comp.f90:66-68).
template <typename T>
__global__ void k_to_aos(const T* __restrict__ q, double* __restrict__ aos, int64_t n, int nf, double g1, int nq,
                         const double* __restrict__ species) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6];
    load_cell(q, n, nf, i, v);
    if (nf == 5) {
      double m2 = (v[1] * v[1]) + (v[2] * v[2]) + (v[3] * v[3]);
      double kin = 0.5 * m2 / v[0];
      double p = g1 * (v[4] - kin);
      v[5] = p / pow(v[0], g1);
    }
#pragma unroll
    for (int f = 0; f < EVORA_NQ; ++f) aos[(int64_t)nq * i + f] = v[f];
    if (species)
      for (int s = 0; s < nq - EVORA_NQ; ++s) aos[(int64_t)nq * i + EVORA_NQ + s] = species[s * n + i];
  }
}

// Deterministic two-pass sum of the six conserved fields.
template <typename T>
__global__ void k_totals_part(const T* __restrict__ q, int64_t n, int nf, int aos, double g1, double* part) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6];
    for (int f = 0; f < 6; ++f) v[f] = 0.0;
    if (aos) {
      for (int f = 0; f < 6; ++f) v[f] = (double)q[6 * i + f];
    } else {
      load_cell(q, n, nf, i, v);
      if (nf == 5) {
        double m2 = (v[1] * v[1]) + (v[2] * v[2]) + (v[3] * v[3]);
        double p = g1 * (v[4] - 0.5 * m2 / v[0]);
        v[5] = p / pow(v[0], g1);
      }
    }
    for (int f = 0; f < 6; ++f) s[f] += v[f];
  }
  __shared__ double red[6][256];
  for (int f = 0; f < 6; ++f) red[f][threadIdx.x] = s[f];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int f = 0; f < 6; ++f) red[f][threadIdx.x] += red[f][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int f = 0; f < 6; ++f) part[6 * blockIdx.x + f] = red[f][0];
}

__global__ void k_totals_final(const double* part, int nb, double* out) {
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[6 * b + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

// One cell of the state (SoA with nf fields, or the reference's AoS) as the
// six FP64 values of q(1:6, cell); S derived as in k_to_aos when not carried.
template <typename T>
__device__ __forceinline__ void cell_load(const T* q, int64_t n, int nf, int aos, double g1, int64_t i,
                                          double v[6]) {
  if (aos) {
    for (int f = 0; f < 6; ++f) v[f] = (double)q[6 * i + f];
    return;
  }
  load_cell(q, n, nf, i, v);
  if (nf == 5) {
    double m2 = (v[1] * v[1]) + (v[2] * v[2]) + (v[3] * v[3]);
    double kin = 0.5 * m2 / v[0];
    double p = g1 * (v[4] - kin);
    v[5] = p / pow(v[0], g1);
  }
}

template <typename T>
__global__ void k_get_plane(const T* __restrict__ q, int64_t n, int nf, int aos, double g1, PlaneMap m,
                            double* __restrict__ out) {
  const int64_t np = (int64_t)m.na * m.nb;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < np; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = m.base + (j % m.na) * m.sa + (j / m.na) * m.sb;
    double v[6];
    cell_load(q, n, nf, aos, g1, i, v);
    for (int f = 0; f < 6; ++f) out[6 * j + f] = v[f];
  }
}

template <typename T>
__global__ void k_set_plane(T* __restrict__ q, int64_t n, int nf, int aos, PlaneMap m,
                            const double* __restrict__ in) {
  const int64_t np = (int64_t)m.na * m.nb;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < np; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = m.base + (j % m.na) * m.sa + (j / m.na) * m.sb;
    if (aos) {
      for (int f = 0; f < 6; ++f) q[6 * i + f] = (T)in[6 * j + f];
    } else {
      for (int f = 0; f < nf; ++f) q[f * n + i] = (T)in[6 * j + f];
    }
  }
}

// snapshot.f90:317-341 per cell: real(q(1)) and real(temp), temp from
// pressure() (comp.f90:45-85, its dual-energy resynchronisation written
// back to the state) and press2temp (comp.f90:87-102, no chemistry).  This
// translation unit is compiled without FMA contraction, so press and temp
// are the reference's FP64 values of the cell.
template <typename T>
__global__ void k_bov(T* __restrict__ q, int64_t n, int nf, int aos, HydroParams P, double temp0,
                      float* __restrict__ dens, float* __restrict__ temp, unsigned* err) {
  const Gas<double> c = Gas<double>::make(P);
  const bool de = P.dualenergy != 0;
  unsigned e = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v[6];
    cell_load(q, n, nf, aos, P.g1, i, v);
    const double press = pressure(v, c, de, e);
    if (de) {
      if (aos) {
        q[6 * i + 4] = (T)v[4];
        q[6 * i + 5] = (T)v[5];
      } else {
        q[4 * n + i] = (T)v[4];
        if (nf == 6) q[5 * n + i] = (T)v[5];
      }
    }
    dens[i] = (float)v[0];
    temp[i] = (float)(press / v[0] * temp0);
  }
  if (e) atomicOr(err, e);
}

}  // namespace

PlaneMap plane_map(const HydroParams& P, int axis, int index0) {
  const int64_t nx = P.nx, nxy = (int64_t)P.nx * P.ny;
  if (axis == 1) return {index0, nx, nxy, P.ny, P.nz};
  if (axis == 2) return {(int64_t)index0 * nx, 1, nxy, P.nx, P.nz};
  return {(int64_t)index0 * nxy, 1, nx, P.nx, P.ny};
}

void state_get_plane(const void* q, bool f32, int64_t n, int nf, int aos, double g1, const PlaneMap& m,
                     double* out, cudaStream_t st) {
  const int64_t np = (int64_t)m.na * m.nb;
  if (f32) k_get_plane<float><<<grid_of(np), 256, 0, st>>>((const float*)q, n, nf, aos, g1, m, out);
  else k_get_plane<double><<<grid_of(np), 256, 0, st>>>((const double*)q, n, nf, aos, g1, m, out);
}

void state_set_plane(void* q, bool f32, int64_t n, int nf, int aos, const PlaneMap& m, const double* in,
                     cudaStream_t st) {
  const int64_t np = (int64_t)m.na * m.nb;
  if (f32) k_set_plane<float><<<grid_of(np), 256, 0, st>>>((float*)q, n, nf, aos, m, in);
  else k_set_plane<double><<<grid_of(np), 256, 0, st>>>((double*)q, n, nf, aos, m, in);
}

void state_bov(void* q, bool f32, int64_t n, int nf, int aos, const HydroParams& P, double temp0, float* dens,
               float* temp, unsigned* err, cudaStream_t st) {
  if (f32) k_bov<float><<<grid_of(n), 256, 0, st>>>((float*)q, n, nf, aos, P, temp0, dens, temp, err);
  else k_bov<double><<<grid_of(n), 256, 0, st>>>((double*)q, n, nf, aos, P, temp0, dens, temp, err);
}

void fused_from_aos(const FusedPlan& pl, const double* aos, void* q, cudaStream_t st, int nq, double* species) {
  if (pl.precision == EVORA_FP32)
    k_from_aos<float><<<grid_of(pl.n), 256, 0, st>>>(aos, (float*)q, pl.n, pl.nf, nq, species);
  else
    k_from_aos<double><<<grid_of(pl.n), 256, 0, st>>>(aos, (double*)q, pl.n, pl.nf, nq, species);
}

void fused_to_aos(const FusedPlan& pl, const void* q, double* aos, cudaStream_t st, int nq, const double* species) {
  if (pl.precision == EVORA_FP32)
    k_to_aos<float><<<grid_of(pl.n), 256, 0, st>>>((const float*)q, aos, pl.n, pl.nf, pl.P.g1, nq, species);
  else
    k_to_aos<double><<<grid_of(pl.n), 256, 0, st>>>((const double*)q, aos, pl.n, pl.nf, pl.P.g1, nq, species);
}

static int totals_run(const void* q, bool f32, int64_t n, int nf, int aos, double g1, double* part, int nb,
                      double out[6], cudaStream_t st) {
  double* fin = part + 6 * nb;   // part holds nb + 1 rows of six
  if (f32) k_totals_part<float><<<nb, 256, 0, st>>>((const float*)q, n, nf, aos, g1, part);
  else k_totals_part<double><<<nb, 256, 0, st>>>((const double*)q, n, nf, aos, g1, part);
  k_totals_final<<<1, 32, 0, st>>>(part, nb, fin);
  cudaError_t e = cudaMemcpyAsync(out, fin, 6 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_cuda_error(e, "totals");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

int fused_totals(const FusedPlan& pl, const void* q, double out[6], cudaStream_t st) {
  return totals_run(q, pl.precision == EVORA_FP32, pl.n, pl.nf, 0, pl.P.g1, pl.partials, pl.nblk_tot, out, st);
}

int fused_totals_aos(const double* aos, int64_t n, double out[6], cudaStream_t st) {
  int64_t nb64 = (n + 255) / 256;
  int nb = (int)(nb64 > 148 * 4 ? 148 * 4 : nb64);
  double* part = nullptr;
  if (cudaMalloc(&part, sizeof(double) * 6 * (nb + 1)) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  int rc = totals_run(aos, false, n, 6, 1, 0.0, part, nb, out, st);
  cudaFree(part);
  return rc;
}

}  // namespace evora
