// abi.cu -- host side of the C ABI: parameters (readparameter defaults,
// compparameter), error reporting, and the drop-in layer entry points that
// mirror primitive / bound / hydrostep / updatetime / compevo / sweep.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/evora_gpu.h"
#include "../../include/evora_io.h"
#include "chem.h"
#include "chemistry.cuh"
#include "common.h"
#include "cosmology.cuh"
#include "dropin_api.h"

namespace evora {

static thread_local char g_last_error[256] = "";

void set_cuda_error(cudaError_t e, const char* where) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s: %s", where, cudaGetErrorString(e));
}

void set_error_message(const char* msg) { std::snprintf(g_last_error, sizeof g_last_error, "%s", msg); }

bool params_to_hydro(const evora_params* p, HydroParams* P, evora_derived* d, int* status) {
  evora_derived dd;
  int rc = evora_compparameter(p, &dd);
  if (status) *status = rc;
  if (rc) return false;
  if (d) *d = dd;
  P->nx = p->nx; P->ny = p->ny; P->nz = p->nz;
  P->solver = p->solver; P->limiter = p->limiter; P->boundtype = p->boundtype;
  P->secondorder = p->secondorder != 0; P->dualenergy = p->dualenergy != 0;
  P->onedimension = dd.onedimension; P->twodimension = dd.twodimension;
  P->g = dd.g; P->g1 = dd.g1; P->g1inv = dd.g1inv; P->gg1 = dd.gg1; P->cfl = dd.cfl;
  P->de_thresh1 = dd.de_thresh1;
  P->dx = dd.dx; P->dy = dd.dy; P->dz = dd.dz;
  P->dxinv = dd.dxinv; P->dyinv = dd.dyinv; P->dzinv = dd.dzinv;
  P->conduction = p->conduction != 0;
  P->simplekappa = p->simplekappa != 0;
  P->c_cond = p->c_cond;
  // comoving coordinates (parameter.f90:227-243)
  P->supercomoving = p->supercomoving != 0;
  P->expansion = p->supercomoving && !p->atomic;
  P->omega0 = p->omega0;
  P->lambda0 = p->lambda0;
  P->c_cosmo = p->c_cosmo;
  P->zstart = p->zstart;
  P->zend = p->zend;
  P->g35 = 3.0 * dd.g - 5.0;
  P->gravc = 1.5 * p->omega0;
  P->fb = p->fb;
  {
    double b[5];
    unit_bases(p, b);
    const double t0 = b[2], l0 = b[3];
    P->u_l02 = l0 * l0;
    P->u_t02 = t0 * t0;
    P->u_m0 = b[4];
    P->u_t03 = std::pow(t0, 3.0);
    P->u_d0 = b[1];
    P->u_l04 = std::pow(l0, 4.0);
    P->u_kcoef = kappa_coef();
    P->u_t0 = t0;
  }
  // chemistry (parameter.f90:95-104: without it, no background, cooling or
  // cooling time step; initchem, chemistry.f90:36-37: chiH = rhoH / mH)
  P->chemistry = p->chemistry != 0;
  P->cooling = p->chemistry && p->cooling;
  P->background = p->chemistry && p->background;
  P->bg = p->bg;
  P->j0 = p->j0;
  P->c_chem = p->c_chem;
  P->substep = p->substep;
  P->chiH = p->rhoh / kMH;
  P->chiHe = p->rhohe / kMHe;
  P->cooldt = P->cooling && p->cooldt;   // parameter.f90:103
  P->noncie = p->chemistry && p->noncie;
  P->c_cooldt = p->c_cooldt;
  // compunits (units.f90:26-73) at the start of the run (a = 1/(1+zstart)
  // with supercomoving, main.f90:58-62)
  evora_units u;
  evora_compunits(p, nullptr, &u);
  P->kappa0 = u.kappa0;
  P->temp0 = u.temp0;
  // pressure floors of chem (chemistry.f90:100-119): temp2press with
  // temp0inv = 1 / temp0, and jeansfloor0 = (dx / jeans0 / c_jeans)^2 when
  // the Jeans floor is on (units.f90:66-71)
  P->tempfloor = p->tempfloor != 0;
  P->jeansfloor = p->jeansfloor != 0;
  P->temp_fl = p->temp_fl;
  P->temp0inv = 1.0 / u.temp0;
  P->jeansfloor0 = u.jeansfloor0;
  return true;
}

void start_time(const evora_params* p, const HydroParams& P, CosmoTime* s) {
  // compparameter: t = tstart, cosmo = 1 (parameter.f90:232-234); then
  // cosmostart with supercomoving (main.f90:58)
  std::memset(s, 0, sizeof *s);
  s->t = p->tstart;
  s->cosmo = 1.0;
  if (p->supercomoving) cosmostart(P, *s);
}

bool is_device_pointer(const void* ptr) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace evora

using namespace evora;

extern "C" {

const char* evora_version(void) { return "evora-b200 0.1 (sm_100a)"; }

}  // extern "C"

namespace {
// out[i] = the FP64 fast reciprocal of x[i], out[n + i] = the device's
// correctly rounded 1.0 / x[i], out[2n + i] = the FP64 fast square root,
// out[3n + i] = the device's correctly rounded sqrt(x[i]).
__global__ void k_selftest_rcp(const double* x, double* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    out[i] = evora::rcp_fast(x[i]);
    out[n + i] = 1.0 / x[i];
    out[2 * n + i] = evora::sqrt_fast(x[i]);
    out[3 * n + i] = sqrt(x[i]);
  }
}
}  // namespace

extern "C" {

int evora_selftest_rcp(const double* x, double* out, int64_t n) {
  if (!x || !out || n <= 0) return EVORA_ERR_ARG;
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, (size_t)n * 5 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int nb = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    k_selftest_rcp<<<nb, 256>>>(d, d + n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + n, (size_t)n * 4 * sizeof(double), cudaMemcpyDeviceToHost);
  if (d) cudaFree(d);
  if (e != cudaSuccess) {
    evora::set_cuda_error(e, "evora_selftest_rcp");
    return EVORA_ERR_CUDA;
  }
  return 0;
}

const char* evora_last_error(void) { return g_last_error; }

void evora_params_default(evora_params* p) {
  std::memset(p, 0, sizeof *p);
  // parameter.f90:43-82 (hydro and grid subset)
  p->secondorder = 1;
  p->solver = 2;
  p->limiter = 1;
  p->cfl = 0.5;
  p->g = (double)1.4f;  // default-real literal
  p->atomic = 0;
  p->nx = p->ny = p->nz = 32;
  p->xmin = 0.0; p->xmax = 1.0;
  p->ymin = 0.0; p->ymax = 1.0;
  p->zmin = 0.0; p->zmax = 1.0;
  p->boundtype = 2;
  p->tstart = 0.0; p->tend = 1.0;
  p->dualenergy = 0;
  p->de_thresh = 0.0;
  p->conduction = 0;
  p->simplekappa = 0;
  p->c_cond = (double)0.1f;
  p->tempfloor = 0;
  p->jeansfloor = 0;
  p->temp_fl = 0.0;
  p->c_jeans = 0.0;
  p->fb = 1.0;
  // parameter.f90:60-65, 82
  p->supercomoving = 0;
  p->c_cosmo = (double)0.1f;
  p->omega0 = 1.0;
  p->lambda0 = 0.0;
  p->hubble0 = 50.0;
  p->box = 1.0;
  p->zstart = 99.0;
  p->zend = 0.0;
  for (int i = 0; i < EVORA_NDUMP; ++i) p->dump_redshift[i] = -1.0;
  // parameter.f90:66-77
  p->chemistry = 0;
  p->noncie = 0;
  p->cooling = 0;
  p->background = 0;
  p->bg = 0;
  p->j0 = 1e-21;
  p->c_chem = (double)0.1f;
  p->substep = (double)0.1f;
  p->rhoh = (double)0.76f;
  p->rhohe = (double)0.24f;
  p->cooldt = 0;
  p->c_cooldt = 0.0;
}

int evora_compparameter(const evora_params* p, evora_derived* d) {
  if (!p || !d) return EVORA_ERR_ARG;
  if (p->nx < 2 || p->ny < 1 || p->nz < 1) return EVORA_ERR_ARG;
  if (p->nz > 1 && p->ny == 1) return EVORA_ERR_ARG;
  if (p->solver != 1 && p->solver != 2) return EVORA_ERR_SOLVER;
  if (p->limiter < 1 || p->limiter > 3) return EVORA_ERR_LIMITER;
  if (p->boundtype < 1 || p->boundtype > 3) return EVORA_ERR_ARG;
  // thermalflux's Spitzer branch (conduction.f90:140-144) reads the electron
  // density that w2n leaves unset without chemistry, and a gradient before
  // it is assigned: only the simplekappa branch is defined in this build
  if (p->conduction && !p->simplekappa) return EVORA_ERR_ARG;
  // chemistry: conduction with chemistry reads the electron density that
  // w2n leaves unset in the CIE build (nw = 5, comp.f90:121-135).  The
  // non-equilibrium build (noncie) is accepted for chem and initchem; the
  // entry points of its 12-field hydro path refuse it.
  if (p->chemistry && p->conduction) return EVORA_ERR_ARG;
  // parameter.f90:164-265
  double g = p->atomic ? (double)(5.0f / 3.0f) : p->g;
  d->g = g;
  d->cfl = p->cfl;
  d->onedimension = (p->ny == 1 && p->nz == 1);
  d->twodimension = (p->nz == 1);
  double xmin = p->xmin, xmax = p->xmax, ymin = p->ymin, ymax = p->ymax;
  double zmin = p->zmin, zmax = p->zmax;
  d->dx = (xmax - xmin) / p->nx;
  d->dy = (ymax - ymin) / p->ny;
  d->dz = (zmax - zmin) / p->nz;
  if (d->onedimension) {
    d->dy = d->dx; d->dz = d->dx;
    ymin = 0.0; ymax = d->dy; zmin = 0.0; zmax = d->dz;
    d->dy = (ymax - ymin) / p->ny;
    d->dz = (zmax - zmin) / p->nz;
  }
  if (d->twodimension) {
    d->dz = d->dx;
    zmin = 0.0; zmax = d->dz;
    d->dz = (zmax - zmin) / p->nz;
  }
  d->dxinv = 1.0 / d->dx; d->dyinv = 1.0 / d->dy; d->dzinv = 1.0 / d->dz;
  d->x0 = xmin + d->dx / 2; d->y0 = ymin + d->dy / 2; d->z0 = zmin + d->dz / 2;
  d->volume = (xmax - xmin) * (ymax - ymin) * (zmax - zmin);
  d->g1 = g - 1.0;
  d->g1inv = 1.0 / d->g1;
  d->gg1 = g / d->g1;
  d->de_thresh1 = p->dualenergy ? 1.0 - p->de_thresh : 1.0;
  if (!(d->dx > 0.0) || !(d->dy > 0.0) || !(d->dz > 0.0)) return EVORA_ERR_ARG;
  return EVORA_OK;
}

void evora_array_sizes(const evora_params* p, int64_t* nq, int64_t* nw, int64_t* ne, int64_t* ns) {
  if (nq) *nq = (int64_t)(p->chemistry ? EVORA_NQ_CHEM : EVORA_NQ) * p->nx * p->ny * p->nz;
  // nw = 11 primitives in the non-equilibrium build (global.f90:29-36)
  const int64_t fw = (p->chemistry && p->noncie) ? 11 : EVORA_NW;
  if (nw) *nw = fw * (p->nx + 4) * (p->ny + 4) * (p->nz + 4);
  if (ne) *ne = fw * (p->nx + 2) * (p->ny + 2) * (p->nz + 2);
  if (ns) *ns = fw * 3 * (p->nx + 2) * (p->ny + 2) * (p->nz + 2);
}

}  // extern "C"

// ------------------------------------------------------------- drop-in --
namespace {

struct DropinState {
  std::mutex mu;
  bool have_params = false;
  evora_params params{};
  HydroParams P{};
  CosmoTime time{};   // module global's time scalars (evora_settime)
  ChemCoef coef{};    // the chemistry's rate coefficients (coef, uv)
  double nH = 0.0, nHe = 0.0;   // module global's nH, nHe (dropin_set_nh)
  int strict = 0;
  int device = -1;
  unsigned* d_err = nullptr;
  unsigned long long* d_smax = nullptr;
  // staging buffers for host arrays: q, w, evo, s
  double* stage[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[4] = {0, 0, 0, 0};
  // resident mode (evora_set_resident): 0 off, EVORA_RESIDENT_FP64 or
  // EVORA_RESIDENT_FP32; the grid holding the state of host array rq
  int resident = 0;
  evora_grid* rgrid = nullptr;
  const double* rq = nullptr;
  bool rq_device_newer = false;   // the grid has steps the host q lacks
  bool rq_host_newer = false;     // host q changed after the upload
};

DropinState& ds() {
  static DropinState s;
  return s;
}

enum { SLOT_Q = 0, SLOT_W = 1, SLOT_E = 2, SLOT_S = 3 };

#define CU(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) {                       \
      set_cuda_error(e_, #call);                   \
      return EVORA_ERR_CUDA;                       \
    }                                              \
  } while (0)

// Resolves a caller pointer to a device pointer: device memory is used in
// place; host memory is copied into a cached staging buffer when copy_in.
int resolve(DropinState& S, int slot, const double* ptr, size_t bytes, bool copy_in, double** out) {
  if (!ptr) return EVORA_ERR_ARG;
  if (is_device_pointer(ptr)) {
    *out = const_cast<double*>(ptr);
    return 0;
  }
  if (S.stage_bytes[slot] < bytes) {
    if (S.stage[slot]) cudaFree(S.stage[slot]);
    S.stage[slot] = nullptr;
    S.stage_bytes[slot] = 0;
    if (cudaMalloc(&S.stage[slot], bytes) != cudaSuccess) {
      cudaGetLastError();
      return EVORA_ERR_NOMEM;
    }
    S.stage_bytes[slot] = bytes;
  }
  if (copy_in) CU(cudaMemcpy(S.stage[slot], ptr, bytes, cudaMemcpyHostToDevice));
  *out = S.stage[slot];
  return 0;
}

int copy_back(double* host, const double* dev, size_t bytes) {
  if (host == dev) return 0;
  CU(cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost));
  return 0;
}

int begin(DropinState& S) {
  if (!S.have_params) return EVORA_ERR_ARG;
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (S.device != dev || !S.d_err) {
    if (S.d_err) cudaFree(S.d_err);
    S.d_err = nullptr;
    // [0]: error word; [8, 32): the three CFL maxima
    CU(cudaMalloc(&S.d_err, 8 + 3 * sizeof(unsigned long long)));
    S.d_smax = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(S.d_err) + 8);
    for (auto& b : S.stage) {
      if (b) cudaFree(b);
      b = nullptr;
    }
    for (auto& n : S.stage_bytes) n = 0;
    S.device = dev;
  }
  CU(cudaMemset(S.d_err, 0, sizeof(unsigned)));
  return 0;
}

int finish(DropinState& S) {
  CU(cudaGetLastError());
  CU(cudaDeviceSynchronize());
  unsigned e = 0;
  CU(cudaMemcpy(&e, S.d_err, sizeof e, cudaMemcpyDeviceToHost));
  return (int)e;
}

// The kernels of the parameters' array layouts (global.f90:30-36).
const DropinOps& ops(const DropinState& S) {
  if (S.P.chemistry && S.P.noncie) return S.strict ? evora::strict::kOpsNcie : evora::fast::kOpsNcie;
  if (S.P.chemistry) return S.strict ? evora::strict::kOpsCie : evora::fast::kOpsCie;
  return S.strict ? evora::strict::kOps : evora::fast::kOps;
}

// ---- resident mode
// The state goes back to host q when the grid has steps q lacks.
int resident_download(DropinState& S) {
  if (!S.rgrid || !S.rq || !S.rq_device_newer) return 0;
  int rc = evora_grid_get_q(S.rgrid, const_cast<double*>(S.rq));
  if (rc) return rc;
  S.rq_device_newer = false;
  return evora_grid_status(S.rgrid);   // errors of the updates since the last wait
}

// Ends the resident grid (after its state went back to the host).
int resident_close(DropinState& S) {
  int rc = resident_download(S);
  if (S.rgrid) evora_grid_destroy(S.rgrid);
  S.rgrid = nullptr;
  S.rq = nullptr;
  S.rq_device_newer = S.rq_host_newer = false;
  return rc;
}

// Binds host q to the resident grid (created on first use with the hydro
// subset of the parameters), uploading q when it is new or changed.
int resident_bind(DropinState& S, const double* q) {
  if (!S.rgrid) {
    evora_params p = S.params;
    // the grid runs only the hydro routines; the physics after the update
    // stays with the drop-in routines of the caller's loop
    p.gravity = 0;
    p.conduction = 0;
    p.tempfloor = p.jeansfloor = 0;
    p.supercomoving = 0;
    p.tend = 1e300;
    const int32_t flags = S.strict ? EVORA_STRICT : 0;
    const int32_t prec = S.resident == EVORA_RESIDENT_FP32 ? EVORA_FP32 : EVORA_FP64;
    int rc = evora_grid_create(&p, prec, flags, &S.rgrid);
    if (rc) {
      S.rgrid = nullptr;
      return rc;
    }
    // the FP32 form's fastest update where it takes the grid (a fixed
    // choice, not timed, so that the results do not depend on a timing)
    if (prec == EVORA_FP32 && !S.strict && (rc = evora_grid_set_tile(S.rgrid, EVORA_FP32_PAIR_TILE))) {
      evora_grid_destroy(S.rgrid);
      S.rgrid = nullptr;
      return rc;
    }
    S.rq = nullptr;
  }
  if (q != S.rq || S.rq_host_newer) {
    if (S.rq && q != S.rq) {
      int rc = resident_download(S);   // the previous array keeps its steps
      if (rc) return rc;
    }
    int rc = evora_grid_set_q(S.rgrid, q);
    if (rc) return rc;
    S.rq = q;
    S.rq_host_newer = S.rq_device_newer = false;
  }
  return 0;
}

}  // namespace

void evora::dropin_resident_read(const double* q) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.resident && q && q == S.rq) resident_download(S);
}

void evora::dropin_resident_write(const double* q) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.resident && q && q == S.rq) {
    resident_download(S);
    S.rq_host_newer = true;
  }
}

bool evora::dropin_params(HydroParams* P) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return false;
  *P = S.P;
  return true;
}

bool evora::dropin_time(CosmoTime* s) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return false;
  *s = S.time;
  return true;
}

bool evora::dropin_coef(ChemCoef* k) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return false;
  *k = S.coef;
  return true;
}

void evora::dropin_set_nh(double nH, double nHe) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  S.nH = nH;
  S.nHe = nHe;
}

bool evora::dropin_nh(double* nH, double* nHe) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return false;
  *nH = S.nH;
  *nHe = S.nHe;
  return true;
}

extern "C" {

int evora_set_params(const evora_params* p) {
  if (!p) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  HydroParams P;
  int rc = 0;
  if (!params_to_hydro(p, &P, nullptr, &rc)) return rc;
  if ((rc = resident_close(S))) return rc;   // a new run: the last state goes home first
  S.params = *p;
  S.P = P;
  start_time(p, P, &S.time);
  start_coef(P, S.time.cosmo, &S.coef);
  S.nH = S.nHe = 0.0;   // a fresh program's module global
  S.have_params = true;
  return 0;
}

int evora_set_strict(int32_t strict) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if ((strict != 0) != (S.strict != 0) && S.rgrid) {
    int rc = resident_close(S);   // the next primitive builds the grid in the new mode
    if (rc) return rc;
  }
  S.strict = strict != 0;
  return 0;
}

int evora_set_resident(int32_t mode) {
  if (mode != 0 && mode != EVORA_RESIDENT_FP64 && mode != EVORA_RESIDENT_FP32) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (mode != S.resident) {
    int rc = resident_close(S);
    if (rc) return rc;
  }
  S.resident = mode;
  return 0;
}

int evora_sync(double* q) {
  if (!q) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.resident || q != S.rq) return 0;
  return resident_download(S);
}

int evora_invalidate(const double* q) {
  if (!q) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.resident && q == S.rq) S.rq_host_newer = true;
  return 0;
}

int evora_primitive(double* w, double* q) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  int rc = begin(S);
  if (rc) return rc;
  if (S.resident) {
    // the primitives are recovered inside the update from the resident
    // state (w is not written); p <= 0 is reported by hydrostep
    if (S.P.chemistry) return EVORA_ERR_ARG;   // resident grids keep q(6) (species apart)
    if (!w || !q || is_device_pointer(q)) return EVORA_ERR_ARG;
    return resident_bind(S, q);
  }
  int64_t nq, nw;
  evora_array_sizes(&S.params, &nq, &nw, nullptr, nullptr);
  double *dq, *dw;
  if ((rc = resolve(S, SLOT_Q, q, nq * 8, true, &dq))) return rc;
  if ((rc = resolve(S, SLOT_W, w, nw * 8, true, &dw))) return rc;
  ops(S).primitive(S.P, dw, dq, S.d_err, nullptr, 0);
  int st = finish(S);
  if (st & EVORA_ERR_CUDA) return st;
  if ((rc = copy_back(w, dw, nw * 8))) return rc;
  if (S.P.dualenergy && (rc = copy_back(q, dq, nq * 8))) return rc;
  return st;
}

int evora_bound(double* w) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  int rc = begin(S);
  if (rc) return rc;
  if (S.resident) return w ? 0 : EVORA_ERR_ARG;   // the ghost map is applied inside the update
  int64_t nw;
  evora_array_sizes(&S.params, nullptr, &nw, nullptr, nullptr);
  double* dw;
  if ((rc = resolve(S, SLOT_W, w, nw * 8, true, &dw))) return rc;
  ops(S).bound(S.P, dw, nullptr, 0);
  int st = finish(S);
  if ((rc = copy_back(w, dw, nw * 8))) return rc;
  return st;
}

int evora_hydrostep(const double* w, double* dt) {
  if (!dt) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  int rc = begin(S);
  if (rc) return rc;
  if (S.resident) {
    if (!w) return EVORA_ERR_ARG;
    if (!S.rgrid || !S.rq) {
      set_error_message("evora_hydrostep: resident mode needs evora_primitive first");
      return EVORA_ERR_ARG;
    }
    double sm[3];
    const int st = grid_cfl_maxima(S.rgrid, sm);
    if (st) return st;
    unsigned e = 0;
    *dt = cfl_dt(S.P, sm[0], sm[1], sm[2], *dt, e);
    return (int)e;
  }
  int64_t nw;
  evora_array_sizes(&S.params, nullptr, &nw, nullptr, nullptr);
  double* dw;
  if ((rc = resolve(S, SLOT_W, w, nw * 8, true, &dw))) return rc;
  CU(cudaMemset(S.d_smax, 0, 3 * sizeof(unsigned long long)));
  ops(S).cfl(S.P, dw, S.d_smax, nullptr, 0);
  int st = finish(S);
  if (st) return st;
  unsigned long long bits[3];
  CU(cudaMemcpy(bits, S.d_smax, sizeof bits, cudaMemcpyDeviceToHost));
  double sm[3];
  std::memcpy(sm, bits, sizeof sm);
  unsigned e = 0;
  *dt = cfl_dt(S.P, sm[0], sm[1], sm[2], *dt, e);
  return (int)e;
}

int evora_updatetime(int32_t* go, int32_t* dump, int32_t* k, double* t, double* dt) {
  (void)dump;
  (void)k;
  if (!go || !t || !dt) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  int g = *go;
  update_time(S.params.tend, *t, *dt, g);
  *go = g;
  return 0;
}

static_assert(sizeof(evora_time) == sizeof(CosmoTime), "evora_time and CosmoTime share one layout");

int evora_cosmostart(evora_time* s) {
  if (!s) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  CosmoTime c;
  start_time(&S.params, S.P, &c);
  std::memcpy(s, &c, sizeof c);
  return 0;
}

int evora_cosmostep(evora_time* s) {
  if (!s) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  CosmoTime c;
  std::memcpy(&c, s, sizeof c);
  unsigned e = 0;
  cosmostep(S.P, c, e);
  std::memcpy(s, &c, sizeof c);
  return (int)e;
}

int evora_compcosmo(evora_time* s) {
  if (!s) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  CosmoTime c;
  std::memcpy(&c, s, sizeof c);
  compcosmo(S.P, c);
  std::memcpy(s, &c, sizeof c);
  return 0;
}

int evora_updatetime_cosmo(int32_t* go, int32_t* dump, int32_t* k, evora_time* s) {
  if (!go || !dump || !k || !s) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  CosmoTime c;
  std::memcpy(&c, s, sizeof c);
  int g = *go, d = *dump;
  unsigned e = 0;
  updatetime(S.P, S.params.tend, S.params.dump_redshift, c, g, d, *k, e);
  std::memcpy(s, &c, sizeof c);
  *go = g;
  *dump = d;
  return (int)e;
}

int evora_initchem(double* q) {
  if (!q) return EVORA_ERR_ARG;
  evora::dropin_resident_write(q);
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params || !S.P.chemistry || is_device_pointer(q)) return EVORA_ERR_ARG;
  // initchem (chemistry.f90:26-70): fully neutral, n(H) = chiH rho,
  // n(He) = chiHe rho, the other species at nfloor; the pressure() call
  // there resynchronises E or S with dual energy
  const HydroParams& P = S.P;
  const int64_t n = (int64_t)P.nx * P.ny * P.nz;
  int rc = 0;
  for (int64_t i = 0; i < n; ++i) {
    double* c = q + (int64_t)EVORA_NQ_CHEM * i;
    const double m2 = (c[1] * c[1]) + (c[2] * c[2]) + (c[3] * c[3]);
    const double kin = 0.5 * m2 / c[0];
    double press;
    if (P.dualenergy && kin / c[4] > P.de_thresh1) {
      press = c[5] * std::pow(c[0], P.g1);
      c[4] = kin + press * P.g1inv;
    } else {
      press = P.g1 * (c[4] - kin);
      if (P.dualenergy) c[5] = press / std::pow(c[0], P.g1);
    }
    if (press <= 0.0) rc |= EVORA_ERR_PRESSURE;
    for (int s = 0; s < 6; ++s) c[EVORA_NQ + s] = kNfloor;
    c[EVORA_NQ + 0] = P.chiH * c[0];
    c[EVORA_NQ + 2] = P.chiHe * c[0];
    S.nH = c[EVORA_NQ + 0];   // module global's nH, nHe: the last cell's stay
    S.nHe = c[EVORA_NQ + 2];
  }
  return rc;
}

int evora_peebles(const evora_time* s, double* fpeebles) {
  if (!s || !fpeebles) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  if (!(s->cosmo > 1e-8)) return EVORA_ERR_ARG;   // the integral starts at a = 1e-8
  *fpeebles = peebles(S.P, s->cosmo);
  return 0;
}

int evora_settime(const evora_time* s) {
  if (!s) return EVORA_ERR_ARG;
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.have_params) return EVORA_ERR_ARG;
  std::memcpy(&S.time, s, sizeof S.time);
  if (S.P.supercomoving) {
    // compunits after compcosmo (main.f90:132-133), with the host's libm
    // power for a^5 (the reference's own)
    evora_units u;
    evora_compunits(&S.params, s, &u);
    S.P.temp0 = u.temp0;
    S.P.temp0inv = 1.0 / u.temp0;
    S.P.kappa0 = u.kappa0;
    if (S.P.chemistry) step_coef(S.P, s->cosmo, s->redshift, &S.coef);   // main.f90:134-135
  }
  return 0;
}

int evora_compevo(const double* w, double* evo, double* s, double dt) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  int rc = begin(S);
  if (rc) return rc;
  if (S.resident) return (w && evo && s) ? 0 : EVORA_ERR_ARG;   // slopes and predictor run inside the update
  int64_t nw, ne, ns;
  evora_array_sizes(&S.params, nullptr, &nw, &ne, &ns);
  double *dw, *de, *dss;
  if ((rc = resolve(S, SLOT_W, w, nw * 8, true, &dw))) return rc;
  if ((rc = resolve(S, SLOT_E, evo, ne * 8, true, &de))) return rc;
  if ((rc = resolve(S, SLOT_S, s, ns * 8, true, &dss))) return rc;
  ops(S).compevo(S.P, dw, de, dss, dt, nullptr, 0);
  int st = finish(S);
  if ((rc = copy_back(evo, de, ne * 8))) return rc;
  if ((rc = copy_back(s, dss, ns * 8))) return rc;
  return st;
}

int evora_sweep(const double* w, double* q, const double* evo, const double* s, double dt) {
  DropinState& S = ds();
  std::lock_guard<std::mutex> lk(S.mu);
  int rc = begin(S);
  if (rc) return rc;
  if (S.resident) {
    if (!w || !evo || !s || !q || S.P.chemistry) return EVORA_ERR_ARG;
    if (!S.rgrid || q != S.rq || S.rq_host_newer) {
      set_error_message("evora_sweep: resident mode needs evora_primitive on this q first");
      return EVORA_ERR_ARG;
    }
    // enqueued without a wait: the errors it raises are returned by the
    // next hydrostep or sync, which wait for the GPU anyway
    const int st = grid_update_dt(S.rgrid, dt, false);
    S.rq_device_newer = true;
    return st;
  }
  int64_t nq, nw, ne, ns;
  evora_array_sizes(&S.params, &nq, &nw, &ne, &ns);
  double *dq, *dw, *de, *dss;
  if ((rc = resolve(S, SLOT_Q, q, nq * 8, true, &dq))) return rc;
  if ((rc = resolve(S, SLOT_W, w, nw * 8, true, &dw))) return rc;
  if ((rc = resolve(S, SLOT_E, evo, ne * 8, true, &de))) return rc;
  if ((rc = resolve(S, SLOT_S, s, ns * 8, true, &dss))) return rc;
  ops(S).sweep(S.P, dw, dq, de, dss, dt, S.d_err, nullptr, 0);
  int st = finish(S);
  if ((rc = copy_back(q, dq, nq * 8))) return rc;
  return st;
}

}  // extern "C"
