// fused.h -- host interface of the fused (structure-of-arrays) backend.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

struct FusedPlan;

// Launches the fused update of one step, qin -> qout.
typedef void (*FusedLaunch)(const FusedPlan& plan, const void* qin, void* qout, GridCtl* ctl,
                            cudaStream_t st);

struct FusedPlan {
  HydroParams P{};
  int precision = 0;   // EVORA_FP64 / EVORA_FP32
  int nf = 5;          // advected fields
  int strict = 0;
  int dim = 3;         // 1, 2 or 3
  int64_t n = 0;       // cells
  int tile = 0;        // entry of the precision's tile table
  int tx = 0, ty = 0, zc = 0;
  int minb = 1;        // CTAs per SM the tile is built for
  size_t smem = 0;
  dim3 grid{1, 1, 1};
  int threads = 0;
  FusedLaunch launch = nullptr;
  void (*cfl)(const FusedPlan&, const void* q, GridCtl* ctl, cudaStream_t st) = nullptr;
  double* partials = nullptr;  // device scratch of the totals reduction
  cudaStream_t alloc_stream = nullptr;  // non-null: partials came from cudaMallocAsync on it
  int nblk_tot = 0;
  // 1: the update also reduces the next step's CFL maxima of the state it
  // writes into ctl->snext (2D and 3D kernels), so that step needs no CFL
  // kernel
  int cfl_fused = 0;
};

// Chooses tiles and the kernel instantiation; allocates small scratch.
// alloc_stream non-null: scratch is allocated stream-ordered on it.
int fused_plan(const HydroParams& P, int precision, int nf, int strict, FusedPlan* plan,
               cudaStream_t alloc_stream = nullptr);
// Number of tile shapes of the plan's precision, and switching between them.
int fused_tiles(const FusedPlan& plan);
void fused_set_tile(FusedPlan* plan, int tile);
void fused_plan_free(FusedPlan* plan);

// hydrostep part 1: per-axis maxima of |u_d| + a into ctl->smax (FP64).
void fused_cfl(const FusedPlan& plan, const void* q, GridCtl* ctl, cudaStream_t st);

// The fused MUSCL-Hancock update (primitive, bound, compevo, sweep).
void fused_update(const FusedPlan& plan, const void* qin, void* qout, GridCtl* ctl, cudaStream_t st);

// Layout conversions between the reference q(6, nx, ny, nz) (FP64) and the
// resident SoA state.  Without the entropy field, q(6) is written as
// p / rho^(g-1) of the current state.
// q(nq, cell) in the reference layout <-> the SoA state; with nq = 12
// (chemistry) q(7:12) <-> `species` (6 FP64 fields, field-major).
void fused_from_aos(const FusedPlan& plan, const double* aos, void* q, cudaStream_t st, int nq = EVORA_NQ,
                    double* species = nullptr);
void fused_to_aos(const FusedPlan& plan, const void* q, double* aos, cudaStream_t st, int nq = EVORA_NQ,
                  const double* species = nullptr);

// Sums of q(1..6) over the grid in FP64, deterministic order (synchronises).
int fused_totals(const FusedPlan& plan, const void* q, double out[6], cudaStream_t st);
int fused_totals_aos(const double* aos, int64_t n, double out[6], cudaStream_t st);

// A plane of cells: cell (a, b), a < na fastest, is linear cell
// base + a * sa + b * sb.
struct PlaneMap {
  int64_t base, sa, sb;
  int na, nb;
};
// axis 1: x plane ix = index0 + 1, 2: y plane, 3: z plane (index0 0-based).
PlaneMap plane_map(const HydroParams& P, int axis, int index0);
// Plane copies between a state (SoA with nf fields, FP32 or FP64, or the
// reference AoS layout when aos != 0) and q(6, plane) in FP64.
void state_get_plane(const void* q, bool f32, int64_t n, int nf, int aos, double g1, const PlaneMap& m,
                     double* out, cudaStream_t st);
void state_set_plane(void* q, bool f32, int64_t n, int nf, int aos, const PlaneMap& m, const double* in,
                     cudaStream_t st);
// Per cell FP32 density and temperature of the brick-of-values snapshot;
// pressure() errors are OR-ed into *err (device).
void state_bov(void* q, bool f32, int64_t n, int nf, int aos, const HydroParams& P, double temp0, float* dens,
               float* temp, unsigned* err, cudaStream_t st);

// One grid of a multi-grid batch (device table): its parameters, its two
// state buffers (par: the one holding the current state), its control
// block, cells, planes per 3D tile, 2 or 3 dimensions, and whether the CFL
// maxima of its current state are in ctl->snext (the previous update reduced
// them) or in ctl->smax (a CFL kernel filled them before the step).
struct MultiGridDesc {
  HydroParams P;
  void* q[2];
  GridCtl* ctl;
  int64_t n;
  int zc, dim, par, fresh;
};
// One work item of a batched update: a tile (bx, by, bz) of grid `grid`.
struct MultiGridItem {
  int grid, bx, by, bz;
};
// meta[0] grids, meta[1] items, meta[2] the next item to take (reset by the
// control kernel of each step).
typedef void (*MultiLaunch)(const MultiGridDesc* grids, const MultiGridItem* items, int* meta, int ctas,
                            cudaStream_t st);

// The multi-grid update of a precision (tile shape, shared memory, threads
// and CTAs per SM of its persistent launch).
MultiLaunch fused_multi_pick(int precision, int strict, int nf, int* tx, int* ty, int* zc, size_t* smem,
                             int* threads, int* ctas_per_sm);

// Instantiation launchers (fused_f64.cu, fused_f64_strict.cu, fused_f32.cu).
#define EVORA_DECLARE_FUSED_NS(ns)                                                           \
  namespace ns {                                                                             \
  FusedLaunch pick(int nf, int dim, int tile, int* tx, int* ty, int* zc, size_t* smem, int* threads, int* minb); \
  int tiles();                                                                               \
  bool tile_fits(const HydroParams& P, int nf, int dim, int tile);                           \
  MultiLaunch multi_pick(int nf, int* tx, int* ty, int* zc, size_t* smem, int* threads, int* ctas_per_sm); \
  void cfl(const FusedPlan& pl, const void* q, GridCtl* ctl, cudaStream_t st);                \
  }
EVORA_DECLARE_FUSED_NS(f64)
EVORA_DECLARE_FUSED_NS(f64s)
EVORA_DECLARE_FUSED_NS(f32)
#undef EVORA_DECLARE_FUSED_NS

}  // namespace evora
