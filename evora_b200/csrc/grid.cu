// grid.cu -- the resident layer: a grid whose state stays in HBM across
// steps.  One step is the hydro subset of the reference loop
// (main.f90:109-155): primitive, bound, hydrostep, updatetime, compevo,
// sweep.  The time scalars live in a device control block (GridCtl) so that a
// step needs no host round trip and can be replayed from a CUDA graph.
//
// Two backends:
//  * fused (default): the conserved state in structure-of-arrays form, one
//    fused kernel per step (fused3d.cu) plus a CFL kernel; FP64 or FP32.
//  * reference kernels (EVORA_REFERENCE_KERNELS): the drop-in layer kernels on
//    device-resident arrays in the reference layouts; FP64 only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <numeric>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/evora_gpu.h"
#include "../../include/evora_io.h"
#include "chemistry.cuh"
#include "common.h"
#include "cosmology.cuh"
#include "dropin_api.h"
#include "fused.h"
#include "gravity.h"
#include "conduction.h"
#include "chem.h"
#include "expansion.h"

using namespace evora;

struct evora_grid {
  evora_params params{};
  evora_derived d{};
  HydroParams P{};
  int precision = EVORA_FP64;
  int flags = 0;
  int device = 0;
  int nf = 5;  // advected fields (5, or 6 with the entropy)
  cudaStream_t stream = nullptr;
  GridCtl* ctl = nullptr;  // device
  // reference-kernel backend
  double* q_aos = nullptr;
  double* w = nullptr;
  double* evo = nullptr;
  double* s = nullptr;
  // fused backend: two SoA copies of the conserved state (ping-pong)
  void* qbuf[2] = {nullptr, nullptr};
  int cur = 0;
  FusedPlan plan{};
  double* aos_stage = nullptr;  // device staging for q in reference layout
  GridCtl ctl_init{};           // host source of the control block set_q uploads
  // kernel timing
  bool timing = false;
  std::vector<cudaEvent_t> events;  // 5 per timed step
  size_t ev_used = 0;
  int64_t launches = 0;
  // multi-step CUDA graphs, key = 4 * steps + 2 * (CFL maxima fresh) +
  // starting buffer
  std::map<long long, cudaGraphExec_t> graphs;
  std::map<long long, int64_t> graph_launches;   // kernel launches per replay, by key
  // the last enqueued step's closing control (step_end) is deferred into the
  // next step's first control kernel or a flush
  bool pending_end = false;
  // the previous update reduced the CFL maxima of the current state into
  // ctl->snext; any other change of the state clears this
  bool cfl_fresh = false;
  // self-gravity after each hydro step (params.gravity)
  bool gravity = false;
  GravPlan grav{};
  // thermal conduction after each step (params.conduction)
  bool conduction = false;
  CondPlan cond{};
  // chem(q) after each step (params.chemistry / tempfloor / jeansfloor)
  bool floors = false;
  // with chemistry: n(H, H+, He, He+, He++, e-), 6 FP64 field-major arrays
  double* species = nullptr;
  // comoving coordinates: expansion terms after each step (params.supercomoving
  // and not atomic)
  bool expansion = false;
  bool async_alloc = false;  // memory from cudaMallocAsync on `stream`
  evora_multigrid* multigrid = nullptr;   // the batch stepping this grid, if any
};

// A batch of resident 2D and 3D grids stepped together: per step one control
// kernel (every grid's hydrostep, updatetime), one persistent update launch
// over the tiles of all grids, one closing control kernel.
struct evora_multigrid {
  int precision = EVORA_FP64;
  int flags = 0;
  int nf = 5;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<evora_grid*> grids;
  bool dirty = true;
  evora::MultiGridDesc* d_desc = nullptr;
  evora::MultiGridItem* d_items = nullptr;
  int* d_meta = nullptr;                   // grids, items, next item
  long long* d_status = nullptr;           // per grid: go | err << 1, then k
  int cap_grids = 0, cap_items = 0;
  evora::MultiLaunch launch = nullptr;
  int tx = 0, ty = 0, zc = 0, threads = 0, ctas = 0;
  size_t smem = 0;
  std::map<int, cudaGraphExec_t> graphs;   // by step count
  long long cell_updates = 0;              // member cells x steps enqueued
};

namespace {

#define CU(call)                 \
  do {                           \
    cudaError_t e_ = (call);     \
    if (e_ != cudaSuccess) {     \
      set_cuda_error(e_, #call); \
      return EVORA_ERR_CUDA;     \
    }                            \
  } while (0)

bool reference_backend(const evora_grid* g) { return (g->flags & EVORA_REFERENCE_KERNELS) != 0; }

int64_t ncells(const evora_grid* g) { return (int64_t)g->P.nx * g->P.ny * g->P.nz; }

size_t elem_size(const evora_grid* g) { return g->precision == EVORA_FP32 ? 4 : 8; }

// use_next 1: the CFL maxima of this step's state were reduced by the
// previous step's update (with the errors that computation raised); 0: a CFL
// kernel fills smax after this; 2: a CFL kernel filled smax before this.
__device__ __forceinline__ void step_begin(GridCtl* ctl, int use_next) {
  if (use_next == 1) {
    ctl->err |= ctl->errnext;
    for (int i = 0; i < 3; ++i) ctl->smax[i] = ctl->snext[i];
  } else if (use_next == 0) {
    ctl->smax[0] = ctl->smax[1] = ctl->smax[2] = 0ull;
  }
  ctl->errnext = 0u;
  ctl->snext[0] = ctl->snext[1] = ctl->snext[2] = 0ull;
  ctl->vcond = ordered_bits(1e99);   // thermalstep's initial v (timestep.f90:82)
  ctl->vcool = ordered_bits(1e6);    // coolstep's initial v (timestep.f90:121)
  // a raised dump holds the grid until the host has read it
  ctl->active = (ctl->go != 0 && ctl->err == 0 && ctl->dump == 0) ? 1 : 0;
}

__global__ void k_step_begin(GridCtl* ctl, int use_next) { step_begin(ctl, use_next); }

// hydrostep part 2 (timestep.f90:26-57), the coolstep and thermalstep
// limits in main.f90:119-121's order, and the master block of
// main.f90:124-137: cosmostep and compcosmo (comoving), updatetime, and
// compunits (comoving).
__device__ __forceinline__ void step_time(const HydroParams& P, GridCtl* ctl) {
  if (!ctl->active || ctl->err) {
    ctl->active = 0;
    return;
  }
  double sm[3];
  for (int i = 0; i < 3; ++i) sm[i] = __longlong_as_double((long long)ctl->smax[i]);
  unsigned e = 0;
  double dt = cfl_dt(P, sm[0], sm[1], sm[2], 1e99, e);
  if (!e && P.cooldt) dt = cool_dt(P.c_cooldt, __longlong_as_double((long long)ctl->vcool), dt, e);
  if (!e && P.conduction) dt = thermal_dt(P, units_of(P, ctl), __longlong_as_double((long long)ctl->vcond), dt, e);
  if (e) {
    ctl->err |= e;
    ctl->active = 0;
    return;
  }
  CosmoTime s{ctl->t, dt, ctl->cosmo, ctl->oldcosmo, ctl->cosmodot, ctl->expand, ctl->redshift};
  if (P.supercomoving) {
    cosmostep(P, s, e);
    if (!e) compcosmo(P, s);
  }
  int go = ctl->go, dump = 0;
  if (!e) updatetime(P, ctl->tend, ctl->dump_redshift, s, go, dump, ctl->k4, e);
  if (e) {
    ctl->err |= e;
    ctl->active = 0;
    return;
  }
  ctl->t = s.t;
  ctl->dt = s.dt;
  ctl->go = go;
  if (P.supercomoving) {
    ctl->cosmo = s.cosmo;
    ctl->oldcosmo = s.oldcosmo;
    ctl->cosmodot = s.cosmodot;
    ctl->expand = s.expand;
    ctl->redshift = s.redshift;
    const Units u = comoving_units(P, s.cosmo);
    ctl->temp0 = u.temp0;
    ctl->temp0inv = u.temp0inv;
    ctl->kappa0 = u.kappa0;
    if (P.chemistry) {   // compbackground and compcoef (main.f90:134-135)
      const double uv = compbackground(P.background, P.bg, P.j0, s.redshift, s.cosmo, ctl->coef.uv);
      compcoef(chem_units(P, s.cosmo), uv, ctl->coef);
    }
    if (dump) {   // main.f90:197-202: dump number k4, then k4 + 1
      ctl->dump = ctl->k4;
      ctl->k4 += 1;
    }
  }
}

__global__ void k_step_time(HydroParams P, GridCtl* ctl) { step_time(P, ctl); }

__device__ __forceinline__ void step_end(GridCtl* ctl) {
  if (ctl->active && ctl->err == 0) ctl->k += 1;
}

__global__ void k_step_end(GridCtl* ctl) { step_end(ctl); }

// The control of consecutive fused steps in one launch: the previous step's
// step_end (when end is set), then this step's step_begin with the maxima
// the previous update reduced, and step_time -- the three single-thread
// kernels' work in their order.
__global__ void k_step_control(HydroParams P, GridCtl* ctl, int end) {
  if (end) step_end(ctl);
  step_begin(ctl, 1);
  step_time(P, ctl);
}

// Control of a multi-grid step, one thread per grid: hydrostep part 2 and
// updatetime (as k_step_begin + k_step_time), and after the update the step
// count, the ping-pong parity and a compact status word.
__global__ void k_mg_begin(MultiGridDesc* g, int* meta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) meta[2] = 0;
  if (i >= meta[0]) return;
  GridCtl* ctl = g[i].ctl;
  step_begin(ctl, g[i].fresh ? 1 : 2);
  g[i].fresh = 1;
  step_time(g[i].P, ctl);
}

__global__ void k_mg_end(MultiGridDesc* g, const int* meta, long long* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= meta[0]) return;
  GridCtl* ctl = g[i].ctl;
  step_end(ctl);
  g[i].par ^= 1;
  status[2 * i] = (long long)(ctl->go != 0) | ((long long)ctl->err << 1);
  status[2 * i + 1] = ctl->k;
}

// An update with the caller's dt (the drop-in layer's resident mode): the
// step is active unless an error was raised; the next step's CFL maxima
// start from zero.
__global__ void k_set_dt(GridCtl* ctl, double dt) {
  ctl->dt = dt;
  ctl->active = ctl->err == 0 ? 1 : 0;
  ctl->errnext = 0u;
  ctl->snext[0] = ctl->snext[1] = ctl->snext[2] = 0ull;
}

// The control block at the start of a run: t = tstart, go, and with
// supercomoving cosmostart's a, da/dt and redshift, the units at that a and
// the first dump index k4 = 1 (main.f90:33, 52-62).
void init_ctl(const evora_grid* g, GridCtl* c) {
  std::memset(c, 0, sizeof *c);
  CosmoTime s;
  start_time(&g->params, g->P, &s);
  c->t = s.t;
  c->tend = g->params.tend;
  c->go = 1;
  c->cosmo = s.cosmo;
  c->oldcosmo = s.oldcosmo;
  c->cosmodot = s.cosmodot;
  c->expand = s.expand;
  c->redshift = s.redshift;
  c->temp0 = g->P.temp0;
  c->temp0inv = g->P.temp0inv;
  c->kappa0 = g->P.kappa0;
  c->k4 = 1;
  std::memcpy(c->dump_redshift, g->params.dump_redshift, sizeof c->dump_redshift);
  if (g->P.chemistry) start_coef(g->P, s.cosmo, &c->coef);
}

// Own kernels of one gravity substep: the mean density (two), the source,
// the Green's function and the integration; the comoving source needs no
// mean.
int grav_launches(const evora_grid* g) { return g->gravity ? (g->grav.comoving ? 3 : 5) : 0; }

// The expansion terms run inside the gravity integration's pass when they
// follow it directly (main.f90:157-178 with neither chem nor conduction).
bool fused_expansion(const evora_grid* g) {
  return g->expansion && g->gravity && !g->floors && !g->conduction && !reference_backend(g);
}

// The expansion terms ride in the default mode's chem(q) pass: chem and the
// expansion are adjacent in main.f90 (167, 178) when there is no conduction.
bool chem_expansion(const evora_grid* g) {
  return g->expansion && g->floors && !g->conduction && !(g->flags & EVORA_STRICT) && !reference_backend(g);
}

void drop_graphs(evora_grid* g) {
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();
  g->graph_launches.clear();
}

cudaEvent_t next_event(evora_grid* g) {
  if (g->ev_used == g->events.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    g->events.push_back(e);
  }
  return g->events[g->ev_used++];
}

void mark(evora_grid* g) {
  if (!g->timing) return;
  cudaEvent_t e = next_event(g);
  if (e) cudaEventRecord(e, g->stream);
}

int enqueue_reference_step(evora_grid* g) {
  const DropinOps& o = (g->flags & EVORA_STRICT) ? evora::strict::kOps : evora::fast::kOps;
  cudaStream_t st = g->stream;
  const int nb = (g->P.nx != 1) + (g->P.ny != 1) + (g->P.nz != 1);
  g->launches += 7 + nb;
  k_step_begin<<<1, 1, 0, st>>>(g->ctl, 0);
  mark(g);
  o.primitive(g->P, g->w, g->q_aos, &g->ctl->err, g->ctl, st);
  o.bound(g->P, g->w, g->ctl, st);
  o.cfl(g->P, g->w, g->ctl->smax, g->ctl, st);
  mark(g);
  k_step_time<<<1, 1, 0, st>>>(g->P, g->ctl);
  mark(g);
  if (g->P.secondorder) o.compevo(g->P, g->w, g->evo, g->s, 0.0, g->ctl, st);
  o.sweep(g->P, g->w, g->q_aos, g->evo, g->s, 0.0, &g->ctl->err, g->ctl, st);
  mark(g);
  if (g->gravity) {
    int rc = grav_potential(g->grav, g->q_aos, false, EVORA_NQ, 1, g->ctl, 1.0);
    if (!rc) rc = grav_integrate(g->grav, g->q_aos, false, EVORA_NQ, 1, g->ctl, 0.0);
    if (rc) return rc;
  }
  mark(g);
  k_step_end<<<1, 1, 0, st>>>(g->ctl);
  CU(cudaGetLastError());
  return 0;
}

// The deferred step_end of the last enqueued step, before the host reads
// the control block or another kind of launch follows.
void flush_step_end(evora_grid* g) {
  if (!g->pending_end) return;
  k_step_end<<<1, 1, 0, g->stream>>>(g->ctl);
  g->launches += 1;
  g->pending_end = false;
}

int enqueue_fused_step(evora_grid* g) {
  cudaStream_t st = g->stream;
  const bool use_next = g->cfl_fresh;
  if (use_next && !g->P.cooldt) {
    // the previous step's end, this step's begin and time in one launch
    k_step_control<<<1, 1, 0, st>>>(g->P, g->ctl, g->pending_end ? 1 : 0);
    g->pending_end = false;
    g->launches += 2;   // the control kernel and the update
    mark(g);
    mark(g);
  } else {
    flush_step_end(g);
    g->launches += use_next ? 3 : 4;
    k_step_begin<<<1, 1, 0, st>>>(g->ctl, use_next ? 1 : 0);
    mark(g);
    if (!use_next) fused_cfl(g->plan, g->qbuf[g->cur], g->ctl, st);
    if (g->P.cooldt) {
      // coolstep (main.f90:120) on the state the step starts from
      int rc =
          cool_step(g->P, g->qbuf[g->cur], g->precision == EVORA_FP32, g->nf, ncells(g), g->species, g->ctl, st);
      if (rc) return rc;
      g->launches += 1;
    }
    mark(g);
    k_step_time<<<1, 1, 0, st>>>(g->P, g->ctl);
  }
  mark(g);
  fused_update(g->plan, g->qbuf[g->cur], g->qbuf[g->cur ^ 1], g->ctl, st);
  mark(g);
  if (g->gravity) {
    // gravpotential + gravintegration on the updated state (main.f90:158-165);
    // with the expansion terms next (no floors or conduction between), they
    // ride in the integration's pass over the cells
    int rc = grav_potential(g->grav, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, 0, g->ctl, 1.0);
    if (!rc)
      rc = grav_integrate(g->grav, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, 0, g->ctl, 0.0,
                          fused_expansion(g) ? &g->P : nullptr);
    if (rc) return rc;
    g->launches += grav_launches(g);   // own kernels; cuFFT adds its own
  }
  if (g->floors) {
    // chem(q): the CIE species and cooling, and the pressure floors (main.f90:167)
    int rc = (g->flags & EVORA_STRICT)
                 ? chem_step(g->P, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, ncells(g), g->species,
                             g->ctl, st)
                 : chem_step_fast(g->P, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, ncells(g),
                                  g->species, g->ctl, st, chem_expansion(g));
    if (rc) return rc;
    g->launches += 1;
  }
  if (g->conduction) {
    // primitive + bound + thermalconduction on the updated state (main.f90:169-175)
    int rc = cond_step(g->cond, g->P, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, g->ctl, 0.0, st);
    if (rc) return rc;
    g->launches += 2;
  }
  if (g->expansion && !fused_expansion(g) && !chem_expansion(g)) {
    // expansion terms of E and S (main.f90:178)
    int rc = expansion_step(g->P, g->qbuf[g->cur ^ 1], g->precision == EVORA_FP32, g->nf, ncells(g), g->ctl, st);
    if (rc) return rc;
    g->launches += 1;
  }
  mark(g);
  g->pending_end = true;   // k_step_end, deferred (flush_step_end, k_step_control)
  CU(cudaGetLastError());
  // The swap is unconditional on the host; an inactive step copies q through
  // unchanged (fused_update does that when the step is inactive).
  g->cur ^= 1;
  g->cfl_fresh = g->plan.cfl_fused != 0;
  return 0;
}

}  // namespace

namespace evora {

int grid_cfl_maxima(evora_grid* g, double smax[3]) {
  if (!g || reference_backend(g)) return EVORA_ERR_ARG;
  cudaStream_t st = g->stream;
  const bool use_next = g->cfl_fresh;
  k_step_begin<<<1, 1, 0, st>>>(g->ctl, use_next ? 1 : 0);
  if (!use_next) fused_cfl(g->plan, g->qbuf[g->cur], g->ctl, st);
  g->launches += use_next ? 1 : 2;
  CU(cudaGetLastError());
  GridCtl c;
  CU(cudaMemcpyAsync(&c, g->ctl, sizeof c, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  for (int i = 0; i < 3; ++i) std::memcpy(&smax[i], &c.smax[i], sizeof(double));
  return (int)c.err;
}

int grid_update_dt(evora_grid* g, double dt, bool sync) {
  if (!g || reference_backend(g)) return EVORA_ERR_ARG;
  cudaStream_t st = g->stream;
  k_set_dt<<<1, 1, 0, st>>>(g->ctl, dt);
  fused_update(g->plan, g->qbuf[g->cur], g->qbuf[g->cur ^ 1], g->ctl, st);
  k_step_end<<<1, 1, 0, st>>>(g->ctl);
  g->launches += 3;
  CU(cudaGetLastError());
  g->cur ^= 1;
  g->cfl_fresh = g->plan.cfl_fused != 0;
  return sync ? evora_grid_status(g) : 0;
}

}  // namespace evora

namespace {

// Device memory of a grid: cudaMalloc, or stream-ordered on the grid's
// stream for grids made by evora_grid_create_async.
cudaError_t dalloc(evora_grid* g, void** p, size_t bytes) {
  return g->async_alloc ? cudaMallocAsync(p, bytes, g->stream) : cudaMalloc(p, bytes);
}
void dfree(evora_grid* g, void* p) {
  if (!p) return;
  if (g->async_alloc) cudaFreeAsync(p, g->stream);
  else cudaFree(p);
}

void free_grid(evora_grid* g) {
  if (!g) return;
  drop_graphs(g);
  for (cudaEvent_t e : g->events) cudaEventDestroy(e);
  fused_plan_free(&g->plan);
  grav_plan_free(&g->grav);
  cond_plan_free(&g->cond);
  dfree(g, g->ctl);
  dfree(g, g->q_aos);
  dfree(g, g->w);
  dfree(g, g->evo);
  dfree(g, g->s);
  dfree(g, g->qbuf[0]);
  dfree(g, g->qbuf[1]);
  dfree(g, g->aos_stage);
  dfree(g, g->species);
  delete g;
}

// Values per cell of q in the reference layout (12 with chemistry).
int nq_of(const evora_grid* g) { return g->params.chemistry ? EVORA_NQ_CHEM : EVORA_NQ; }
}  // namespace

namespace evora {

int grid_set_q_async(evora_grid* g, const double* q) {
  int64_t nq;
  evora_array_sizes(&g->params, &nq, nullptr, nullptr, nullptr);
  const bool dev = is_device_pointer(q);
  if (reference_backend(g)) {
    CU(cudaMemcpyAsync(g->q_aos, q, nq * 8, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       g->stream));
  } else {
    const double* src = q;
    if (!dev) {
      if (!g->aos_stage) CU(dalloc(g, (void**)&g->aos_stage, nq * 8));
      CU(cudaMemcpyAsync(g->aos_stage, q, nq * 8, cudaMemcpyHostToDevice, g->stream));
      src = g->aos_stage;
    }
    g->cur = 0;
    fused_from_aos(g->plan, src, g->qbuf[0], g->stream, nq_of(g), g->species);
  }
  g->cfl_fresh = false;
  if (g->multigrid) g->multigrid->dirty = true;   // its table entry (parity, maxima) changes
  init_ctl(g, &g->ctl_init);
  CU(cudaMemcpyAsync(g->ctl, &g->ctl_init, sizeof(GridCtl), cudaMemcpyHostToDevice, g->stream));
  return 0;
}

int grid_get_q_async(evora_grid* g, double* q) {
  int64_t nq;
  evora_array_sizes(&g->params, &nq, nullptr, nullptr, nullptr);
  const bool dev = is_device_pointer(q);
  if (reference_backend(g)) {
    CU(cudaMemcpyAsync(q, g->q_aos, nq * 8, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       g->stream));
  } else {
    double* dst = q;
    if (!dev) {
      if (!g->aos_stage) CU(dalloc(g, (void**)&g->aos_stage, nq * 8));
      dst = g->aos_stage;
    }
    fused_to_aos(g->plan, g->qbuf[g->cur], dst, g->stream, nq_of(g), g->species);
    if (!dev) CU(cudaMemcpyAsync(q, dst, nq * 8, cudaMemcpyDeviceToHost, g->stream));
  }
  return 0;
}

}  // namespace evora

namespace {

int create_grid(const evora_params* p, int32_t precision, int32_t flags, cudaStream_t astream, evora_grid** out);
int graph_steps(evora_grid* g, int nsteps);

}  // namespace

extern "C" {

int evora_grid_create(const evora_params* p, int32_t precision, int32_t flags, evora_grid** out) {
  return create_grid(p, precision, flags, nullptr, out);
}

int evora_grid_create_async(const evora_params* p, int32_t precision, int32_t flags, void* stream,
                            evora_grid** out) {
  if (!stream) return EVORA_ERR_ARG;
  return create_grid(p, precision, flags, (cudaStream_t)stream, out);
}

}  // extern "C"

namespace {

int create_grid(const evora_params* p, int32_t precision, int32_t flags, cudaStream_t astream, evora_grid** out) {
  if (!p || !out) return EVORA_ERR_ARG;
  *out = nullptr;
  if (precision != EVORA_FP64 && precision != EVORA_FP32) return EVORA_ERR_ARG;
  evora_grid* g = new (std::nothrow) evora_grid();
  if (!g) return EVORA_ERR_NOMEM;
  int rc = 0;
  if (!params_to_hydro(p, &g->P, &g->d, &rc)) {
    delete g;
    return rc;
  }
  g->params = *p;
  g->precision = precision;
  g->flags = flags;
  g->nf = (flags & EVORA_CARRY_ENTROPY) || p->dualenergy ? 6 : 5;
  if (reference_backend(g) && precision != EVORA_FP64) {
    delete g;
    return EVORA_ERR_ARG;
  }
  cudaGetDevice(&g->device);
  g->stream = astream;
  g->async_alloc = astream != nullptr;
  if (dalloc(g, (void**)&g->ctl, sizeof(GridCtl)) != cudaSuccess) goto nomem;
  if (reference_backend(g)) {
    int64_t nq, nw, ne, ns;
    evora_array_sizes(p, &nq, &nw, &ne, &ns);
    if (dalloc(g, (void**)&g->q_aos, nq * 8) != cudaSuccess) goto nomem;
    if (dalloc(g, (void**)&g->w, nw * 8) != cudaSuccess) goto nomem;
    if (dalloc(g, (void**)&g->evo, ne * 8) != cudaSuccess) goto nomem;
    if (dalloc(g, (void**)&g->s, ns * 8) != cudaSuccess) goto nomem;
    if (cudaMemsetAsync(g->w, 0, nw * 8, g->stream) != cudaSuccess) goto nomem;
    if (cudaMemsetAsync(g->evo, 0, ne * 8, g->stream) != cudaSuccess) goto nomem;  // main.f90:76-77
    if (cudaMemsetAsync(g->s, 0, ns * 8, g->stream) != cudaSuccess) goto nomem;
  } else {
    size_t bytes = (size_t)g->nf * ncells(g) * elem_size(g);
    if (dalloc(g, &g->qbuf[0], bytes) != cudaSuccess) goto nomem;
    if (dalloc(g, &g->qbuf[1], bytes) != cudaSuccess) goto nomem;
    rc = fused_plan(g->P, g->precision, g->nf, (flags & EVORA_STRICT) != 0, &g->plan, astream);
    if (rc) {
      free_grid(g);
      return rc;
    }
  }
  if (p->chemistry || p->tempfloor || p->jeansfloor) {
    // the non-equilibrium build advects the species through the update
    // (nf = 12); grids advect 5 or 6 fields
    if (reference_backend(g) || (p->chemistry && p->noncie)) {
      free_grid(g);
      return EVORA_ERR_ARG;   // chem(q) runs on the resident SoA state
    }
    g->floors = true;
    g->plan.cfl_fused = 0;     // the state changes after the update
    if (p->chemistry && dalloc(g, (void**)&g->species, sizeof(double) * 6 * ncells(g)) != cudaSuccess) goto nomem;
  }
  if (p->conduction) {
    if (reference_backend(g)) {
      free_grid(g);
      return EVORA_ERR_ARG;   // conduction runs on the resident SoA state
    }
    g->conduction = true;
    g->plan.cfl_fused = 0;     // the state changes after the update
    rc = cond_plan(ncells(g), &g->cond);
    if (rc) {
      free_grid(g);
      return rc;
    }
  }
  if (p->gravity) {
    // the potential changes the state after the update: the next step's
    // CFL maxima come from the CFL kernel, not from the update
    g->gravity = true;
    g->plan.cfl_fused = 0;
    rc = grav_plan(g->P, &g->grav, g->stream);
    if (rc) {
      free_grid(g);
      return rc;
    }
  }
  if (p->supercomoving) {
    if (reference_backend(g)) {
      free_grid(g);
      return EVORA_ERR_ARG;   // the comoving terms run on the resident SoA state
    }
    g->expansion = g->P.expansion != 0;
    g->plan.cfl_fused = 0;     // the expansion terms change the state after the update
  }
  {
    GridCtl c;
    init_ctl(g, &c);
    if (cudaMemcpyAsync(g->ctl, &c, sizeof c, cudaMemcpyHostToDevice, g->stream) != cudaSuccess) goto nomem;
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) goto nomem;
  }
  *out = g;
  return 0;
nomem:
  cudaGetLastError();
  free_grid(g);
  return EVORA_ERR_NOMEM;
}

}  // namespace

extern "C" {

int evora_grid_destroy(evora_grid* g) {
  if (!g) return EVORA_ERR_ARG;
  if (g->multigrid) evora_multigrid_remove(g->multigrid, g);
  if (g->async_alloc) {
    free_grid(g);   // stream-ordered frees: no device-wide synchronisation
    return 0;
  }
  if (g->stream) cudaStreamSynchronize(g->stream);
  else cudaDeviceSynchronize();
  free_grid(g);
  return 0;
}

int evora_grid_set_stream(evora_grid* g, void* stream) {
  if (!g) return EVORA_ERR_ARG;
  if (g->async_alloc && (cudaStream_t)stream != g->stream) return EVORA_ERR_ARG;  // memory is ordered on it
  drop_graphs(g);
  g->stream = (cudaStream_t)stream;
  if (g->gravity) grav_set_stream(&g->grav, g->stream);
  return 0;
}

int evora_grid_set_q(evora_grid* g, const double* q) {
  if (!g || !q) return EVORA_ERR_ARG;
  int rc = grid_set_q_async(g, q);
  if (rc) return rc;
  CU(cudaStreamSynchronize(g->stream));
  return 0;
}

int evora_grid_get_q(evora_grid* g, double* q) {
  if (!g || !q) return EVORA_ERR_ARG;
  int rc = grid_get_q_async(g, q);
  if (rc) return rc;
  CU(cudaStreamSynchronize(g->stream));
  return 0;
}

int evora_grid_step(evora_grid* g, int32_t nsteps, int32_t sync) {
  if (!g || nsteps < 0) return EVORA_ERR_ARG;
  if (g->multigrid) {
    set_error_message("evora_grid_step: the grid is stepped by its multi-grid batch");
    return EVORA_ERR_ARG;
  }
  // Several steps on a capturable stream replay graphs of at most 32 steps
  // (instantiating a graph costs with its node count; replays are cheap).
  while (g->stream != nullptr && nsteps >= 2 && !g->timing) {
    const int chunk = nsteps < 32 ? nsteps : 32;
    int rc = graph_steps(g, chunk);
    if (rc) return rc;
    nsteps -= chunk;
  }
  for (int i = 0; i < nsteps; ++i) {
    int rc = reference_backend(g) ? enqueue_reference_step(g) : enqueue_fused_step(g);
    if (rc) return rc;
  }
  flush_step_end(g);
  CU(cudaGetLastError());
  if (sync) return evora_grid_status(g);
  return 0;
}

}  // extern "C"

namespace {

int graph_steps(evora_grid* g, int nsteps) {
  {
    // Steps replayed from a CUDA graph (cached per step count and starting
    // buffer); the step kernels read dt and the active flag from the device
    // control block, so a graph is valid for any time of the run.
    const int start = g->cur;
    const bool fresh = g->cfl_fresh;
    const long long key = 4LL * nsteps + (fresh ? 2 : 0) + start;
    auto it = g->graphs.find(key);
    if (it == g->graphs.end()) {
      cudaGraph_t graph;
      CU(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
      int rc = 0;
      const int64_t launches0 = g->launches;
      for (int i = 0; i < nsteps && !rc; ++i)
        rc = reference_backend(g) ? enqueue_reference_step(g) : enqueue_fused_step(g);
      if (!rc) flush_step_end(g);
      cudaError_t e = cudaStreamEndCapture(g->stream, &graph);
      g->pending_end = false;
      g->cur = start;
      g->cfl_fresh = fresh;
      const int64_t per_replay = g->launches - launches0;
      g->launches = launches0;
      if (rc) return rc;
      if (e != cudaSuccess) {
        set_cuda_error(e, "cudaStreamEndCapture");
        return EVORA_ERR_CUDA;
      }
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        set_cuda_error(e, "cudaGraphInstantiate");
        return EVORA_ERR_CUDA;
      }
      it = g->graphs.emplace(key, ex).first;
      g->graph_launches[key] = per_replay;
    }
    CU(cudaGraphLaunch(it->second, g->stream));
    g->launches += g->graph_launches[key];   // the kernels the capture enqueued
    if (!reference_backend(g)) {
      g->cur = start ^ (nsteps & 1);
      g->cfl_fresh = g->plan.cfl_fused != 0;
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int evora_grid_time(evora_grid* g, double* t, double* dt, int32_t* go, int64_t* k) {
  if (!g) return EVORA_ERR_ARG;
  GridCtl c;
  CU(cudaMemcpyAsync(&c, g->ctl, sizeof c, cudaMemcpyDeviceToHost, g->stream));
  CU(cudaStreamSynchronize(g->stream));
  if (t) *t = c.t;
  if (dt) *dt = c.dt;
  if (go) *go = c.go;
  if (k) *k = c.k;
  return 0;
}

int evora_grid_cosmo(evora_grid* g, evora_time* s, int32_t* dump) {
  if (!g) return EVORA_ERR_ARG;
  GridCtl c;
  CU(cudaMemcpyAsync(&c, g->ctl, sizeof c, cudaMemcpyDeviceToHost, g->stream));
  CU(cudaStreamSynchronize(g->stream));
  if (s) {
    s->t = c.t;
    s->dt = c.dt;
    s->cosmo = c.cosmo;
    s->oldcosmo = c.oldcosmo;
    s->cosmodot = c.cosmodot;
    s->expand = c.expand;
    s->redshift = c.redshift;
  }
  if (dump) *dump = c.dump;
  if (c.dump) {
    const int zero = 0;
    CU(cudaMemcpyAsync(&g->ctl->dump, &zero, sizeof zero, cudaMemcpyHostToDevice, g->stream));
    CU(cudaStreamSynchronize(g->stream));
  }
  return 0;
}

int evora_grid_status(evora_grid* g) {
  if (!g) return EVORA_ERR_ARG;
  GridCtl c;
  cudaError_t e = cudaMemcpyAsync(&c, g->ctl, sizeof c, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    set_cuda_error(e, "evora_grid_status");
    return EVORA_ERR_CUDA;
  }
  return (int)c.err;
}

int evora_grid_autotune(evora_grid* g, int32_t reps, int32_t* chosen, double* ms_per_tile, int32_t max_tiles) {
  if (!g || reps < 1) return EVORA_ERR_ARG;
  if (reference_backend(g)) {
    if (chosen) *chosen = 0;
    return 0;
  }
  const int nt = fused_tiles(g->plan);
  drop_graphs(g);
  // Save the control block, compute this step's dt, then time each tile's
  // update from the current buffer into the other one; the current state is
  // untouched and the control block is restored afterwards.
  GridCtl saved;
  CU(cudaMemcpyAsync(&saved, g->ctl, sizeof saved, cudaMemcpyDeviceToHost, g->stream));
  CU(cudaStreamSynchronize(g->stream));
  k_step_begin<<<1, 1, 0, g->stream>>>(g->ctl, 0);
  fused_cfl(g->plan, g->qbuf[g->cur], g->ctl, g->stream);
  k_step_time<<<1, 1, 0, g->stream>>>(g->P, g->ctl);
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  int best = g->plan.tile;
  double best_ms = 1e300;
  for (int t = 0; t < nt; ++t) {
    fused_set_tile(&g->plan, t);
    fused_update(g->plan, g->qbuf[g->cur], g->qbuf[g->cur ^ 1], g->ctl, g->stream);  // warm-up
    CU(cudaEventRecord(e0, g->stream));
    for (int r = 0; r < reps; ++r) fused_update(g->plan, g->qbuf[g->cur], g->qbuf[g->cur ^ 1], g->ctl, g->stream);
    CU(cudaEventRecord(e1, g->stream));
    CU(cudaEventSynchronize(e1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    const double per = ms / reps;
    if (ms_per_tile && t < max_tiles) ms_per_tile[t] = per;
    if (per < best_ms) {
      best_ms = per;
      best = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fused_set_tile(&g->plan, best);
  CU(cudaMemcpyAsync(g->ctl, &saved, sizeof saved, cudaMemcpyHostToDevice, g->stream));
  CU(cudaStreamSynchronize(g->stream));
  CU(cudaGetLastError());
  if (chosen) *chosen = best;
  return 0;
}

int evora_grid_set_tile(evora_grid* g, int32_t tile) {
  if (!g) return EVORA_ERR_ARG;
  if (reference_backend(g)) return tile == 0 ? 0 : EVORA_ERR_ARG;
  if (tile < 0 || tile >= fused_tiles(g->plan)) return EVORA_ERR_ARG;
  drop_graphs(g);
  fused_set_tile(&g->plan, tile);
  return 0;
}

int evora_grid_set_timing(evora_grid* g, int32_t on) {
  if (!g) return EVORA_ERR_ARG;
  g->timing = on != 0;
  g->ev_used = 0;
  g->launches = 0;
  return 0;
}

int evora_grid_timing_split(evora_grid* g, double* cfl_ms, double* update_ms, double* physics_ms, int64_t* steps,
                            int64_t* launches) {
  if (!g) return EVORA_ERR_ARG;
  CU(cudaStreamSynchronize(g->stream));
  // 5 events per timed step: begin | CFL | control | update | physics | end
  double up = 0.0, cf = 0.0, ph = 0.0;
  const size_t nstep = g->ev_used / 5;
  for (size_t i = 0; i < nstep; ++i) {
    float a = 0.f, b = 0.f, c = 0.f;
    CU(cudaEventElapsedTime(&a, g->events[5 * i + 0], g->events[5 * i + 1]));
    CU(cudaEventElapsedTime(&b, g->events[5 * i + 2], g->events[5 * i + 3]));
    CU(cudaEventElapsedTime(&c, g->events[5 * i + 3], g->events[5 * i + 4]));
    cf += a;
    up += b;
    ph += c;
  }
  if (cfl_ms) *cfl_ms = cf;
  if (update_ms) *update_ms = up;
  if (physics_ms) *physics_ms = ph;
  if (steps) *steps = (int64_t)nstep;
  if (launches) *launches = g->launches;
  g->ev_used = 0;
  g->launches = 0;
  return 0;
}

int evora_grid_timing(evora_grid* g, double* update_ms, double* cfl_ms, int64_t* steps, int64_t* launches) {
  double up = 0.0, ph = 0.0;
  const int rc = evora_grid_timing_split(g, cfl_ms, &up, &ph, steps, launches);
  if (!rc && update_ms) *update_ms = up + ph;
  return rc;
}

static int plane_args(evora_grid* g, int32_t axis, int32_t index, PlaneMap* m) {
  if (!g || axis < 1 || axis > 3) return EVORA_ERR_ARG;
  const int extent = axis == 1 ? g->P.nx : (axis == 2 ? g->P.ny : g->P.nz);
  if (index < 1 || index > extent) return EVORA_ERR_ARG;
  *m = plane_map(g->P, axis, index - 1);
  return 0;
}

// Plane copies through a device staging buffer when the caller's memory is
// on the host (stream-ordered allocation on the grid's stream).
int evora_grid_get_plane(evora_grid* g, int32_t axis, int32_t index, double* out) {
  PlaneMap m;
  int rc = plane_args(g, axis, index, &m);
  if (rc || !out) return rc ? rc : EVORA_ERR_ARG;
  const size_t bytes = sizeof(double) * 6 * (size_t)m.na * m.nb;
  const bool dev = is_device_pointer(out);
  double* dst = out;
  if (!dev) CU(cudaMallocAsync((void**)&dst, bytes, g->stream));
  const bool ref = reference_backend(g);
  state_get_plane(ref ? (const void*)g->q_aos : g->qbuf[g->cur], !ref && g->precision == EVORA_FP32, ncells(g),
                  g->nf, ref ? 1 : 0, g->P.g1, m, dst, g->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !dev) e = cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, g->stream);
  if (!dev) cudaFreeAsync(dst, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    set_cuda_error(e, "evora_grid_get_plane");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

int evora_grid_set_plane(evora_grid* g, int32_t axis, int32_t index, const double* in) {
  PlaneMap m;
  int rc = plane_args(g, axis, index, &m);
  if (rc || !in) return rc ? rc : EVORA_ERR_ARG;
  const size_t bytes = sizeof(double) * 6 * (size_t)m.na * m.nb;
  const bool dev = is_device_pointer(in);
  double* src = const_cast<double*>(in);
  if (!dev) CU(cudaMallocAsync((void**)&src, bytes, g->stream));
  cudaError_t e = dev ? cudaSuccess : cudaMemcpyAsync(src, in, bytes, cudaMemcpyHostToDevice, g->stream);
  const bool ref = reference_backend(g);
  g->cfl_fresh = false;   // the state changed under the reduced CFL maxima
  if (e == cudaSuccess) {
    state_set_plane(ref ? (void*)g->q_aos : g->qbuf[g->cur], !ref && g->precision == EVORA_FP32, ncells(g), g->nf,
                    ref ? 1 : 0, m, src, g->stream);
    e = cudaGetLastError();
  }
  if (!dev) cudaFreeAsync(src, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    set_cuda_error(e, "evora_grid_set_plane");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

int evora_grid_totals(evora_grid* g, double out[6]) {
  if (!g || !out) return EVORA_ERR_ARG;
  if (reference_backend(g)) {
    return fused_totals_aos(g->q_aos, ncells(g), out, g->stream);
  }
  return fused_totals(g->plan, g->qbuf[g->cur], out, g->stream);
}

}  // extern "C"

namespace evora {

const evora_params* grid_params(const evora_grid* g) { return &g->params; }

int grid_bov(evora_grid* g, double temp0, float* dens, float* temp) {
  const int64_t n = ncells(g);
  float* d = nullptr;
  unsigned* err = nullptr;
  CU(cudaMallocAsync((void**)&d, sizeof(float) * 2 * n + 16, g->stream));
  err = reinterpret_cast<unsigned*>(d + 2 * n);
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), g->stream);
  const bool ref = reference_backend(g);
  g->cfl_fresh = false;   // pressure() may resynchronise E or S in place
  if (e == cudaSuccess) {
    state_bov(ref ? (void*)g->q_aos : g->qbuf[g->cur], !ref && g->precision == EVORA_FP32, n, g->nf, ref ? 1 : 0,
              g->P, temp0, d, d + n, err, g->stream);
    e = cudaGetLastError();
  }
  unsigned herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dens, d, sizeof(float) * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(temp, d + n, sizeof(float) * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, g->stream);
  cudaFreeAsync(d, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) {
    set_cuda_error(e, "snapshot fields");
    return EVORA_ERR_CUDA;
  }
  return (int)herr;
}

}  // namespace evora

// ------------------------------------------------------ multi-grid batches --
namespace {

int mg_rebuild(evora_multigrid* m) {
  const int n = (int)m->grids.size();
  std::vector<MultiGridDesc> desc(n);
  std::vector<MultiGridItem> items3, items2;
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  // larger grids first, so that the last items of a step are small ones
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
    const evora_grid* ga = m->grids[a];
    const evora_grid* gb = m->grids[b];
    return (int64_t)ga->P.nx * ga->P.ny * ga->P.nz > (int64_t)gb->P.nx * gb->P.ny * gb->P.nz;
  });
  for (int i = 0; i < n; ++i) {
    evora_grid* g = m->grids[i];
    MultiGridDesc& d = desc[i];
    d.P = g->P;
    d.q[0] = g->qbuf[0];
    d.q[1] = g->qbuf[1];
    d.ctl = g->ctl;
    d.n = ncells(g);
    d.dim = g->plan.dim;
    d.zc = d.dim == 3 ? std::min(m->zc, g->P.nz) : 1;
    d.par = g->cur;
    d.fresh = g->cfl_fresh ? 1 : 0;
  }
  for (int i : idx) {
    const MultiGridDesc& d = desc[i];
    const int gx = (d.P.nx + m->tx - 1) / m->tx, gy = (d.P.ny + m->ty - 1) / m->ty;
    const int gz = d.dim == 3 ? (d.P.nz + d.zc - 1) / d.zc : 1;
    auto& dst = d.dim == 3 ? items3 : items2;
    for (int bz = 0; bz < gz; ++bz)
      for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx) dst.push_back(MultiGridItem{i, bx, by, bz});
  }
  items3.insert(items3.end(), items2.begin(), items2.end());   // 3D items (ZC planes) before 2D ones
  const int ni = (int)items3.size();
  if (n > m->cap_grids || ni > m->cap_items) {
    CU(cudaStreamSynchronize(m->stream));
    for (auto& kv : m->graphs) cudaGraphExecDestroy(kv.second);
    m->graphs.clear();
    if (n > m->cap_grids) {
      cudaFree(m->d_desc);
      cudaFree(m->d_status);
      m->d_desc = nullptr;
      m->d_status = nullptr;
      const int cap = std::max(2 * n, 64);
      CU(cudaMalloc(&m->d_desc, sizeof(MultiGridDesc) * cap));
      CU(cudaMalloc(&m->d_status, sizeof(long long) * 2 * cap));
      m->cap_grids = cap;
    }
    if (ni > m->cap_items) {
      cudaFree(m->d_items);
      m->d_items = nullptr;
      const int cap = std::max(2 * ni, 4096);
      CU(cudaMalloc(&m->d_items, sizeof(MultiGridItem) * cap));
      m->cap_items = cap;
    }
  }
  const int meta[3] = {n, ni, 0};
  if (n) CU(cudaMemcpyAsync(m->d_desc, desc.data(), sizeof(MultiGridDesc) * n, cudaMemcpyHostToDevice, m->stream));
  if (ni) CU(cudaMemcpyAsync(m->d_items, items3.data(), sizeof(MultiGridItem) * ni, cudaMemcpyHostToDevice, m->stream));
  CU(cudaMemcpyAsync(m->d_meta, meta, sizeof meta, cudaMemcpyHostToDevice, m->stream));
  // grids without the CFL maxima of their state get them from the CFL kernel
  for (evora_grid* g : m->grids)
    if (!g->cfl_fresh) {
      k_step_begin<<<1, 1, 0, m->stream>>>(g->ctl, 0);
      fused_cfl(g->plan, g->qbuf[g->cur], g->ctl, m->stream);
    }
  CU(cudaGetLastError());
  // the host copies above must stay alive until enqueued work has read them
  CU(cudaStreamSynchronize(m->stream));
  m->dirty = false;
  return 0;
}

void mg_enqueue(evora_multigrid* m, int nsteps) {
  const int cb = (m->cap_grids + 127) / 128;
  for (int k = 0; k < nsteps; ++k) {
    k_mg_begin<<<cb, 128, 0, m->stream>>>(m->d_desc, m->d_meta);
    m->launch(m->d_desc, m->d_items, m->d_meta, m->ctas, m->stream);
    k_mg_end<<<cb, 128, 0, m->stream>>>(m->d_desc, m->d_meta, m->d_status);
  }
}

bool mg_accepts(const evora_multigrid* m, const evora_grid* g) {
  return !reference_backend(g) && g->precision == m->precision &&
         (g->flags & ~EVORA_REFERENCE_KERNELS) == m->flags && g->nf == m->nf && g->plan.dim >= 2 &&
         !g->gravity && !g->conduction && !g->floors && !g->expansion && !g->P.supercomoving &&
         !g->P.chemistry && !g->P.cooldt;
}

}  // namespace

extern "C" {

int evora_multigrid_create(int32_t precision, int32_t flags, void* stream, evora_multigrid** out) {
  if (!out || (precision != EVORA_FP32 && precision != EVORA_FP64)) return EVORA_ERR_ARG;
  if (flags & EVORA_REFERENCE_KERNELS) return EVORA_ERR_ARG;
  *out = nullptr;
  evora_multigrid* m = new (std::nothrow) evora_multigrid();
  if (!m) return EVORA_ERR_NOMEM;
  m->precision = precision;
  m->flags = flags;
  m->nf = (flags & EVORA_CARRY_ENTROPY) ? 6 : 5;
  m->stream = (cudaStream_t)stream;
  cudaGetDevice(&m->device);
  int per_sm = 1, sms = 148;
  m->launch = fused_multi_pick(precision, (flags & EVORA_STRICT) != 0, m->nf, &m->tx, &m->ty, &m->zc, &m->smem,
                               &m->threads, &per_sm);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  m->ctas = sms * per_sm;
  if (cudaMalloc(&m->d_meta, sizeof(int) * 4) != cudaSuccess) {
    cudaGetLastError();
    delete m;
    return EVORA_ERR_NOMEM;
  }
  *out = m;
  return 0;
}

int evora_multigrid_destroy(evora_multigrid* m) {
  if (!m) return EVORA_ERR_ARG;
  cudaStreamSynchronize(m->stream);
  for (evora_grid* g : m->grids) g->multigrid = nullptr;
  for (auto& kv : m->graphs) cudaGraphExecDestroy(kv.second);
  cudaFree(m->d_desc);
  cudaFree(m->d_items);
  cudaFree(m->d_meta);
  cudaFree(m->d_status);
  delete m;
  return 0;
}

int evora_multigrid_add(evora_multigrid* m, evora_grid* g) {
  if (!m || !g || g->multigrid) return EVORA_ERR_ARG;
  if (!mg_accepts(m, g)) {
    set_error_message("evora_multigrid_add: a member is a 2D or 3D fused grid of the batch's precision and "
                      "flags with no physics after the update");
    return EVORA_ERR_ARG;
  }
  CU(cudaStreamSynchronize(g->stream));   // its set-up work is done
  m->grids.push_back(g);
  g->multigrid = m;
  m->dirty = true;
  return 0;
}

int evora_multigrid_remove(evora_multigrid* m, evora_grid* g) {
  if (!m || !g || g->multigrid != m) return EVORA_ERR_ARG;
  CU(cudaStreamSynchronize(m->stream));   // no batch work touches it any more
  m->grids.erase(std::find(m->grids.begin(), m->grids.end(), g));
  g->multigrid = nullptr;
  m->dirty = true;
  return 0;
}

int evora_multigrid_step(evora_multigrid* m, int32_t nsteps, int32_t sync) {
  if (!m || nsteps < 0) return EVORA_ERR_ARG;
  if (m->dirty) {
    int rc = mg_rebuild(m);
    if (rc) return rc;
  }
  if (m->grids.empty() || nsteps == 0) return 0;
  int left = nsteps;
  while (left > 0) {
    const int chunk = left < 32 ? left : 32;
    if (m->stream) {
      auto it = m->graphs.find(chunk);
      if (it == m->graphs.end()) {
        cudaGraph_t graph;
        CU(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        mg_enqueue(m, chunk);
        cudaError_t e = cudaStreamEndCapture(m->stream, &graph);
        if (e != cudaSuccess) {
          set_cuda_error(e, "evora_multigrid_step: capture");
          return EVORA_ERR_CUDA;
        }
        cudaGraphExec_t exec;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          set_cuda_error(e, "evora_multigrid_step: instantiate");
          return EVORA_ERR_CUDA;
        }
        it = m->graphs.emplace(chunk, exec).first;
      }
      CU(cudaGraphLaunch(it->second, m->stream));
    } else {
      mg_enqueue(m, chunk);
    }
    left -= chunk;
  }
  CU(cudaGetLastError());
  for (evora_grid* g : m->grids) {
    if (nsteps & 1) g->cur ^= 1;
    g->cfl_fresh = g->plan.cfl_fused != 0;
    g->launches += 3LL * nsteps;
    m->cell_updates += (long long)nsteps * ncells(g);
  }
  if (sync) CU(cudaStreamSynchronize(m->stream));
  return 0;
}

int evora_multigrid_status(evora_multigrid* m, evora_grid** grids, int32_t* go, uint32_t* err, int64_t* k,
                           int32_t max, int32_t* n) {
  if (!m || !n || max < 0) return EVORA_ERR_ARG;
  CU(cudaStreamSynchronize(m->stream));
  const int cnt = std::min<int>(max, (int)m->grids.size());
  *n = cnt;
  if (cnt == 0) return 0;
  if (m->dirty) {
    // not stepped since the last change: read the members' own control blocks
    for (int i = 0; i < cnt; ++i) {
      double t, dt;
      int32_t g_go;
      int64_t g_k;
      int rc = evora_grid_time(m->grids[i], &t, &dt, &g_go, &g_k);
      if (rc) return rc;
      if (grids) grids[i] = m->grids[i];
      if (go) go[i] = g_go;
      if (err) err[i] = (uint32_t)evora_grid_status(m->grids[i]);
      if (k) k[i] = g_k;
    }
    return 0;
  }
  std::vector<long long> st(2 * (size_t)cnt);
  CU(cudaMemcpy(st.data(), m->d_status, sizeof(long long) * 2 * cnt, cudaMemcpyDeviceToHost));
  for (int i = 0; i < cnt; ++i) {
    if (grids) grids[i] = m->grids[i];
    if (go) go[i] = (int32_t)(st[2 * i] & 1);
    if (err) err[i] = (uint32_t)(st[2 * i] >> 1);
    if (k) k[i] = st[2 * i + 1];
  }
  return 0;
}

}  // extern "C"
