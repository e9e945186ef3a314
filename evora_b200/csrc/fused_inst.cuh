// fused_inst.cuh -- one arithmetic instantiation of the fused backend: the
// update kernels for NF = 5/6 fields and 1, 2, 3 dimensions, and the CFL
// kernel, compiled with this translation unit's floating-point flags.
// Requires EVORA_FNS (namespace), EVORA_T (state type) and the tile shape
// EVORA_TX, EVORA_TY, EVORA_ZC.
#pragma once

#include <cudaTypedefs.h>

#include "batch_kernel.cuh"
#include "conduction.h"
#include "fused.h"
#include "fused_kernel.cuh"
#include "fused_tma.cuh"
#if EVORA_PRECISION_F32
#include "fused_pair.cuh"
#endif

namespace evora {
namespace EVORA_FNS {

using TT = EVORA_T;

// Tile table of this precision: (TX, TY, ZC, CTAs per SM, TMA, PIPE).
// TMA = 1: the tensor-staged 3D kernel of fused_tma.cuh, for grids tiled by
// whole tiles (the plan falls back to entry 0 elsewhere).  PIPE = 1: the
// two-barrier pipelined 3D march of fused_kernel.cuh (FP32; in FP64 it
// measured no faster than the three-barrier march, 3.24 against 3.23 ms per
// 256^3 launch).  Entry 0 is the
// default for grids the TMA kernel does not take; evora_grid_autotune times
// all entries on the grid itself.  The 3D kernels are instantiated for every
// entry, the 1D and 2D ones for entry 0 only.
template <int I> struct Tile;
#if EVORA_PRECISION_F32
template <> struct Tile<0> { static constexpr int TX = 32, TY = 8, ZC = 32, MINB = 3, TMA = 0, PIPE = 1; };
template <> struct Tile<1> { static constexpr int TX = 16, TY = 16, ZC = 32, MINB = 3, TMA = 0, PIPE = 1; };
template <> struct Tile<2> { static constexpr int TX = 32, TY = 8, ZC = 32, MINB = 2, TMA = 0, PIPE = 1; };
template <> struct Tile<3> { static constexpr int TX = 16, TY = 8, ZC = 32, MINB = 4, TMA = 0, PIPE = 1; };
template <> struct Tile<4> { static constexpr int TX = 32, TY = 8, ZC = 32, MINB = 2, TMA = 1, PIPE = 1; };
// two cells per thread on packed FP32 pairs (fused_pair.cuh)
template <> struct Tile<5> { static constexpr int TX = 32, TY = 8, ZC = 32, MINB = 3, TMA = 2, PIPE = 1; };
constexpr int kTiles = 6;
#else
template <> struct Tile<0> { static constexpr int TX = 16, TY = 8, ZC = 32, MINB = 3, TMA = 0, PIPE = 0; };
template <> struct Tile<1> { static constexpr int TX = 32, TY = 4, ZC = 32, MINB = 3, TMA = 0, PIPE = 0; };
template <> struct Tile<2> { static constexpr int TX = 16, TY = 8, ZC = 16, MINB = 3, TMA = 0, PIPE = 0; };
template <> struct Tile<3> { static constexpr int TX = 16, TY = 8, ZC = 64, MINB = 3, TMA = 0, PIPE = 0; };
template <> struct Tile<4> { static constexpr int TX = 16, TY = 8, ZC = 32, MINB = 2, TMA = 1, PIPE = 0; };
constexpr int kTiles = 5;
#endif

// The shared-memory layout of the k_fused kernel of entry C.
template <class C, int NF>
using TileSmem = FusedSmem<TT, NF, C::TX, C::TY, kSmemDq<TT, C::PIPE != 0>>;

// cuTensorMapEncodeTiled from the driver (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The 4D map (x, y, z, field) of an SoA state q[f][z][y][x] with a box of
// one halo'd plane of all fields, as fused_tma.cuh stages it.
template <int NF, int TX, int TY>
bool encode_state_map(const HydroParams& P, const void* q, CUtensorMap* map) {
  using S = TmaSmem<TT, NF, TX, TY>;
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nz, (cuuint64_t)NF};
  const cuuint64_t es = sizeof(TT);
  const cuuint64_t strides[3] = {es * P.nx, es * P.nx * P.ny, es * P.nx * P.ny * P.nz};
  const cuuint32_t box[4] = {(cuuint32_t)S::SX, (cuuint32_t)S::RY, 1, (cuuint32_t)NF};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, sizeof(TT) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         4, const_cast<void*>(q), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Whether the TMA kernel of this shape takes the grid: whole tiles in x and
// y, a 3D grid, 16-byte aligned rows.
template <int TX, int TY>
bool tma_fits(const HydroParams& P, int dim) {
  return dim == 3 && P.nx % TX == 0 && P.ny % TY == 0 && ((size_t)P.nx * sizeof(TT)) % 16 == 0;
}

template <int NF, int DIM, int I>
void launch(const FusedPlan& pl, const void* qin, void* qout, GridCtl* ctl, cudaStream_t st) {
  FusedArgs<TT> A{pl.P, (const TT*)qin, (TT*)qout, ctl, pl.n, pl.cfl_fused, pl.zc};
  if constexpr (DIM == 1) {
    k_fused1d<TT, NF><<<pl.grid, pl.threads, 0, st>>>(A);
  } else {
    using C = Tile<I>;
#if EVORA_PRECISION_F32
    if constexpr (C::TMA == 2 && DIM == 3 && NF == 5) {
      CUtensorMap map;
      if (encode_state_map<5, C::TX, C::TY>(pl.P, qin, &map)) {
        k_fused_pair<C::TX, C::TY, C::ZC, C::MINB><<<pl.grid, pl.threads, pl.smem, st>>>(A, map);
        return;
      }
      k_fused<TT, NF, DIM, C::TX, C::TY, C::ZC, 2, C::PIPE != 0>
          <<<pl.grid, C::TX * C::TY, sizeof(TileSmem<C, NF>), st>>>(A);
      return;
    }
#endif
    if constexpr (C::TMA == 1 && DIM == 3) {
      CUtensorMap map;
      if (encode_state_map<NF, C::TX, C::TY>(pl.P, qin, &map)) {
        k_fused_tma<TT, NF, C::TX, C::TY, C::ZC, C::MINB><<<pl.grid, pl.threads, pl.smem, st>>>(A, map);
        return;
      }
      // the map was checked at plan time; should it fail here, the same
      // tile runs without tensor staging
      k_fused<TT, NF, DIM, C::TX, C::TY, C::ZC, C::MINB, C::PIPE != 0>
          <<<pl.grid, pl.threads, sizeof(TileSmem<C, NF>), st>>>(A);
    } else {
      k_fused<TT, NF, DIM, C::TX, C::TY, C::ZC, C::MINB, C::PIPE != 0><<<pl.grid, pl.threads, pl.smem, st>>>(A);
    }
  }
}

template <int NF, int DIM, int I>
FusedLaunch pick_one(int* tx, int* ty, int* zc, size_t* smem, int* threads, int* minb) {
  if constexpr (DIM == 1) {
    *tx = 128; *ty = 1; *zc = 1; *smem = 0; *threads = 128; *minb = 1;
  } else {
    using C = Tile<I>;
    *tx = C::TX; *ty = C::TY; *zc = DIM == 3 ? C::ZC : 1; *minb = C::MINB;
    *smem = sizeof(TileSmem<C, NF>);
    *threads = C::TX * C::TY;
    auto k = k_fused<TT, NF, DIM, C::TX, C::TY, C::ZC, C::TMA == 2 ? 2 : C::MINB, C::PIPE != 0>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
#if EVORA_PRECISION_F32
    if constexpr (C::TMA == 2 && DIM == 3 && NF == 5) {
      *smem = sizeof(PairSmem<float, C::TX, C::TY>);
      *threads = C::TX / 2 * C::TY;
      auto kp = k_fused_pair<C::TX, C::TY, C::ZC, C::MINB>;
      cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
      cudaFuncSetAttribute(kp, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
#endif
    if constexpr (C::TMA == 1 && DIM == 3) {
      *smem = sizeof(TmaSmem<TT, NF, C::TX, C::TY>);
      auto kt = k_fused_tma<TT, NF, C::TX, C::TY, C::ZC, C::MINB>;
      cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
      cudaFuncSetAttribute(kt, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
  }
  return &launch<NF, DIM, I>;
}

int tiles() { return kTiles; }

// Whether tile entry `tile` can run this grid (TMA entries need whole tiles
// and an encodable tensor map).
bool tile_fits(const HydroParams& P, int nf, int dim, int tile) {
#if EVORA_PRECISION_F32
  if (tile == 5) {
    using C5 = Tile<5>;
    if (nf != 5 || !pair_config(P) || !tma_fits<C5::TX, C5::TY>(P, dim)) return false;
    CUtensorMap map;
    return encode_state_map<5, C5::TX, C5::TY>(P, reinterpret_cast<const void*>((uintptr_t)1 << 20), &map);
  }
#endif
  if (tile != 4) return true;
  using C = Tile<4>;
  if (!tma_fits<C::TX, C::TY>(P, dim)) return false;
  // encode against an aligned dummy address: only shapes and strides are checked
  CUtensorMap map;
  const void* fake = reinterpret_cast<const void*>((uintptr_t)1 << 20);
  return nf == 5 ? encode_state_map<5, C::TX, C::TY>(P, fake, &map) : encode_state_map<6, C::TX, C::TY>(P, fake, &map);
}

FusedLaunch pick(int nf, int dim, int tile, int* tx, int* ty, int* zc, size_t* smem, int* threads, int* minb) {
  if (nf == 5 && dim == 3) {
    switch (tile) {
      case 1: return pick_one<5, 3, 1>(tx, ty, zc, smem, threads, minb);
      case 2: return pick_one<5, 3, 2>(tx, ty, zc, smem, threads, minb);
      case 3: return pick_one<5, 3, 3>(tx, ty, zc, smem, threads, minb);
      case 4: return pick_one<5, 3, 4>(tx, ty, zc, smem, threads, minb);
#if EVORA_PRECISION_F32
      case 5: return pick_one<5, 3, 5>(tx, ty, zc, smem, threads, minb);
#endif
      default: return pick_one<5, 3, 0>(tx, ty, zc, smem, threads, minb);
    }
  }
  if (nf == 5) {
    if (dim == 1) return pick_one<5, 1, 0>(tx, ty, zc, smem, threads, minb);
    return pick_one<5, 2, 0>(tx, ty, zc, smem, threads, minb);
  }
  if (dim == 1) return pick_one<6, 1, 0>(tx, ty, zc, smem, threads, minb);
  if (dim == 2) return pick_one<6, 2, 0>(tx, ty, zc, smem, threads, minb);
  switch (tile) {
    case 1: return pick_one<6, 3, 1>(tx, ty, zc, smem, threads, minb);
    case 2: return pick_one<6, 3, 2>(tx, ty, zc, smem, threads, minb);
    case 3: return pick_one<6, 3, 3>(tx, ty, zc, smem, threads, minb);
    case 4: return pick_one<6, 3, 4>(tx, ty, zc, smem, threads, minb);
    default: return pick_one<6, 3, 0>(tx, ty, zc, smem, threads, minb);
  }
}

// ---- multi-grid batches: one persistent launch updates the tiles of many
// 2D and 3D grids of uneven sizes (the tile program of entry 0), pulling
// (grid, tile) items from an atomic work queue; each grid keeps its own dt,
// control block and ping-pong parity (MultiGridDesc).
template <int NF>
__global__ void __launch_bounds__(Tile<0>::TX* Tile<0>::TY, Tile<0>::MINB)
    k_multi(const MultiGridDesc* grids, const MultiGridItem* items, int* meta) {
  using C = Tile<0>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& sm = *reinterpret_cast<FusedSmem<TT, NF, C::TX, C::TY>*>(smem_raw);
  __shared__ __align__(16) unsigned char a_raw[sizeof(FusedArgs<TT>)];
  __shared__ int s_item, s_dim, s_bx, s_by, s_bz;
  auto& A = *reinterpret_cast<FusedArgs<TT>*>(a_raw);
  const int nitems = meta[1];
  for (;;) {
    if (threadIdx.x == 0) {
      const int it = atomicAdd(&meta[2], 1);
      s_item = it;
      if (it < nitems) {
        const MultiGridItem w = items[it];
        const MultiGridDesc& d = grids[w.grid];
        A.P = d.P;
        A.qin = (const TT*)d.q[d.par];
        A.qout = (TT*)d.q[d.par ^ 1];
        A.ctl = d.ctl;
        A.n = d.n;
        A.cfl_next = 1;
        A.zc = d.zc;
        s_dim = d.dim;
        s_bx = w.bx;
        s_by = w.by;
        s_bz = w.bz;
      }
    }
    __syncthreads();
    if (s_item >= nitems) break;
    if (s_dim == 3) fused_tile<TT, NF, 3, C::TX, C::TY, C::ZC>(A, sm, threadIdx.x, s_bx, s_by, s_bz);
    else fused_tile<TT, NF, 2, C::TX, C::TY, C::ZC>(A, sm, threadIdx.x, s_bx, s_by, 0);
    __syncthreads();   // the shared state is reused by the next item
  }
}

template <int NF>
void multi_launch(const MultiGridDesc* grids, const MultiGridItem* items, int* meta, int ctas, cudaStream_t st) {
  using C = Tile<0>;
  k_multi<NF><<<ctas, C::TX * C::TY, sizeof(FusedSmem<TT, NF, C::TX, C::TY>), st>>>(grids, items, meta);
}

MultiLaunch multi_pick(int nf, int* tx, int* ty, int* zc, size_t* smem, int* threads, int* ctas_per_sm) {
  using C = Tile<0>;
  *tx = C::TX;
  *ty = C::TY;
  *zc = C::ZC;
  *threads = C::TX * C::TY;
  *ctas_per_sm = C::MINB;
  if (nf == 5) {
    *smem = sizeof(FusedSmem<TT, 5, C::TX, C::TY>);
    cudaFuncSetAttribute(k_multi<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
    cudaFuncSetAttribute(k_multi<5>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return &multi_launch<5>;
  }
  *smem = sizeof(FusedSmem<TT, 6, C::TX, C::TY>);
  cudaFuncSetAttribute(k_multi<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
  cudaFuncSetAttribute(k_multi<6>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  return &multi_launch<6>;
}

// hydrostep part 1 on the SoA state: maxima of |u_d| + a (per cell in the
// working precision, cfl_speeds; maxima and dt in FP64).
template <int NF>
__global__ void k_cfl_soa(HydroParams P, const TT* __restrict__ q, int64_t n, GridCtl* ctl) {
  if (ctl_skip(ctl)) return;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, vmin = 1e99;
  unsigned err = 0;
  const Units U = units_of(P, ctl);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    TT qv[6], s[3];
#pragma unroll
    for (int f = 0; f < NF; ++f) qv[f] = __ldg(q + f * n + i);
    cfl_speeds<TT, NF>(qv, P, P.dualenergy != 0, err, s);
    const double s0 = s[0], s1 = s[1], s2 = s[2];
    if (s0 > m0) m0 = s0;
    if (s1 > m1) m1 = s1;
    if (s2 > m2) m2 = s2;
    if (P.conduction) {
      // thermalstep (timestep.f90:84-93): min over cells of rho / kappa
      double qd[6], w[5];
#pragma unroll
      for (int f = 0; f < NF; ++f) qd[f] = (double)qv[f];
      q2w(qd, w, Gas<double>::make(P), P.dualenergy != 0, err);
      const double v = kFast ? thermal_v_fast(U, w[0], w[4]) : thermal_v(U, w[0], w[4]);
      if (v < vmin) vmin = v;
    }
  }
  if (P.conduction) {
    for (int off = 16; off > 0; off >>= 1) vmin = fmin2(vmin, __shfl_xor_sync(0xffffffffu, vmin, off));
    if ((threadIdx.x & 31) == 0) atomicMin(&ctl->vcond, ordered_bits(vmin));
  }
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
      atomicMax(&ctl->smax[0], ordered_bits(m0));
      atomicMax(&ctl->smax[1], ordered_bits(m1));
      atomicMax(&ctl->smax[2], ordered_bits(m2));
    }
  }
  if (err) atomicOr(&ctl->err, err);
}

void cfl(const FusedPlan& pl, const void* q, GridCtl* ctl, cudaStream_t st) {
  int64_t blocks = (pl.n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (pl.nf == 5) k_cfl_soa<5><<<(int)blocks, 256, 0, st>>>(pl.P, (const TT*)q, pl.n, ctl);
  else k_cfl_soa<6><<<(int)blocks, 256, 0, st>>>(pl.P, (const TT*)q, pl.n, ctl);
}

// ---- batched tubes
template <int NF, int NT>
void batch_launch(const BatchPlan& pl, void* q, cudaStream_t st) {
  BatchArgs<TT> A;
  A.P = pl.P;
  A.xmin = pl.xmin;
  A.xmax = pl.xmax;
  A.q = (TT*)q;
  A.ntot = pl.ntot;
  A.tubes = pl.tubes;
  A.order = pl.order;
  A.ntubes = pl.ntubes;
  A.head = pl.head;
  A.budget = pl.budget;
  A.quantum = pl.quantum;
  A.cap = pl.cap;
  A.capw = pl.capw;
  A.gscratch = (TT*)pl.gscratch;
  A.nmax = pl.nmax;
  A.cell_updates = pl.cell_updates;
  k_tubes<TT, NF, NT><<<pl.ctas, NT, pl.smem, st>>>(A);
}

template <int NF, int NT>
BatchLaunch batch_pick_one(BatchPlan* pl) {
  pl->threads = NT;
  pl->smem = ((size_t)NF * pl->cap + 5 * ((size_t)pl->cap + 4)) * sizeof(TT);
  pl->capw = std::max(pl->cap, (int)(pl->smem / (5 * sizeof(TT))) - 4);
  auto k = k_tubes<TT, NF, NT>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl->smem);
  cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  return &batch_launch<NF, NT>;
}

BatchLaunch batch_pick(int nf, int threads, BatchPlan* pl) {
  if (nf == 5) {
    if (threads == 128) return batch_pick_one<5, 128>(pl);
    if (threads == 512) return batch_pick_one<5, 512>(pl);
    return batch_pick_one<5, 256>(pl);
  }
  if (threads == 128) return batch_pick_one<6, 128>(pl);
  if (threads == 512) return batch_pick_one<6, 512>(pl);
  return batch_pick_one<6, 256>(pl);
}

template <int NF, int NT>
int max_ctas_one(size_t smem) {
  int nb = 0;
  cudaFuncSetAttribute(k_tubes<TT, NF, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tubes<TT, NF, NT>, NT, smem);
  return nb;
}

int batch_max_ctas_per_sm(int nf, int threads, size_t smem) {
  if (nf == 5) {
    if (threads == 128) return max_ctas_one<5, 128>(smem);
    if (threads == 512) return max_ctas_one<5, 512>(smem);
    return max_ctas_one<5, 256>(smem);
  }
  if (threads == 128) return max_ctas_one<6, 128>(smem);
  if (threads == 512) return max_ctas_one<6, 512>(smem);
  return max_ctas_one<6, 256>(smem);
}

}  // namespace EVORA_FNS
}  // namespace evora
