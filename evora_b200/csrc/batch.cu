// batch.cu -- host side of the batched-tube layer (evora_batch_*): many
// independent 1D tubes, each with its own length, time and end time,
// advanced by one persistent kernel launch (batch_kernel.cuh).  Repeated
// launches with a fixed step budget are replayed from CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/evora_gpu.h"
#include "batch.h"
#include "common.h"

using namespace evora;

struct evora_batch {
  evora_params params{};
  HydroParams P{};
  int precision = EVORA_FP32;
  int flags = 0;
  int nf = 5;
  int strict = 0;
  int ntubes = 0;
  std::vector<int> n;
  std::vector<long long> offset;
  std::vector<double> work;     // queue order estimate
  std::vector<double> tend;
  long long ntot = 0;
  int nmax = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void* q = nullptr;
  TubeState* tubes = nullptr;
  int* order = nullptr;
  int* head = nullptr;
  unsigned long long* cell_updates = nullptr;
  double* aos_stage = nullptr;
  size_t aos_bytes = 0;
  void* gscratch = nullptr;
  size_t gscratch_bytes = 0;
  BatchPlan plan{};
  BatchLaunch launch = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  bool order_dirty = true;
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

size_t esize(const evora_batch* b) { return b->precision == EVORA_FP32 ? 4 : 8; }

BatchLaunch (*pick_fn(const evora_batch* b))(int, int, BatchPlan*) {
  if (b->precision == EVORA_FP32) return f32::batch_pick;
  return b->strict ? f64s::batch_pick : f64::batch_pick;
}
int (*occ_fn(const evora_batch* b))(int, int, size_t) {
  if (b->precision == EVORA_FP32) return f32::batch_max_ctas_per_sm;
  return b->strict ? f64s::batch_max_ctas_per_sm : f64::batch_max_ctas_per_sm;
}

void drop_graphs(evora_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}

// cap: tubes up to this length are staged in shared memory.
int configure(evora_batch* b, int threads, int cap) {
  drop_graphs(b);
  BatchPlan& pl = b->plan;
  pl.P = b->P;
  pl.xmin = b->params.xmin;
  pl.xmax = b->params.xmax;
  pl.nf = b->nf;
  pl.ntot = b->ntot;
  pl.tubes = b->tubes;
  pl.order = b->order;
  pl.ntubes = b->ntubes;
  pl.head = b->head;
  pl.cell_updates = b->cell_updates;
  pl.nmax = b->nmax;
  pl.cap = std::max(2, std::min(cap, b->nmax));
  b->launch = pick_fn(b)(b->nf, threads, &pl);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = occ_fn(b)(b->nf, threads, pl.smem);
  if (per_sm < 1) return EVORA_ERR_ARG;
  pl.ctas = std::max(1, std::min(b->ntubes, sms * per_sm));
  if (b->nmax > pl.cap) {
    size_t need = (size_t)pl.ctas * (size_t)(b->nf + 5) * (size_t)(b->nmax + 4) * esize(b);
    if (need > b->gscratch_bytes) {
      cudaFree(b->gscratch);
      b->gscratch = nullptr;
      b->gscratch_bytes = 0;
      if (cudaMalloc(&b->gscratch, need) != cudaSuccess) {
        cudaGetLastError();
        return EVORA_ERR_NOMEM;
      }
      b->gscratch_bytes = need;
    }
  }
  pl.gscratch = b->gscratch;
  return 0;
}

// Largest shared-memory capacity (cells) that keeps `ctas_per_sm` CTAs.
int cap_for(const evora_batch* b, int ctas_per_sm) {
  const size_t per_sm = 227 * 1024;
  const size_t budget = per_sm / ctas_per_sm - 2048;   // static shared + reserve
  const size_t per_cell = (size_t)(b->nf + 5) * esize(b);
  long long cap = (long long)(budget / per_cell) - 4;
  return (int)std::max(2LL, cap);
}

int upload_order(evora_batch* b) {
  std::vector<int> ord(b->ntubes);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return b->work[a] > b->work[c]; });
  CU(cudaMemcpyAsync(b->order, ord.data(), sizeof(int) * ord.size(), cudaMemcpyHostToDevice, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  b->order_dirty = false;
  return 0;
}

template <typename T>
__global__ void k_tube_from_aos(const double* __restrict__ aos, T* __restrict__ q, long long ntot, long long off,
                                long long n, int nf) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    for (int f = 0; f < nf; ++f) q[f * ntot + off + i] = (T)aos[EVORA_NQ * i + f];
}

template <typename T>
__global__ void k_tube_to_aos(const T* __restrict__ q, double* __restrict__ aos, long long ntot, long long off,
                              long long n, int nf, double g1) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v[6];
    for (int f = 0; f < nf; ++f) v[f] = (double)q[f * ntot + off + i];
    if (nf == 5) {   // q(6) = p / rho^(g-1) of the current state
      double m2 = (v[1] * v[1]) + (v[2] * v[2]) + (v[3] * v[3]);
      double p = g1 * (v[4] - 0.5 * m2 / v[0]);
      v[5] = p / pow(v[0], g1);
    }
    for (int f = 0; f < EVORA_NQ; ++f) aos[EVORA_NQ * i + f] = v[f];
  }
}

int grid_of(long long n) {
  long long g = (n + 255) / 256;
  return (int)std::max(1LL, std::min(g, 148LL * 8));
}

}  // namespace

void evora::tube_from_aos(const double* aos, void* q, bool f32, long long ntot, long long off, long long n, int nf,
                          cudaStream_t st) {
  if (f32) k_tube_from_aos<float><<<grid_of(n), 256, 0, st>>>(aos, (float*)q, ntot, off, n, nf);
  else k_tube_from_aos<double><<<grid_of(n), 256, 0, st>>>(aos, (double*)q, ntot, off, n, nf);
}

void evora::tube_to_aos(const void* q, double* aos, bool f32, long long ntot, long long off, long long n, int nf,
                        double g1, cudaStream_t st) {
  if (f32) k_tube_to_aos<float><<<grid_of(n), 256, 0, st>>>((const float*)q, aos, ntot, off, n, nf, g1);
  else k_tube_to_aos<double><<<grid_of(n), 256, 0, st>>>((const double*)q, aos, ntot, off, n, nf, g1);
}

evora::BatchLaunch evora::batch_pick_for(int precision, int strict, int nf, int threads, BatchPlan* pl) {
  if (precision == EVORA_FP32) return f32::batch_pick(nf, threads, pl);
  return strict ? f64s::batch_pick(nf, threads, pl) : f64::batch_pick(nf, threads, pl);
}

int evora::batch_ctas_per_sm(int precision, int strict, int nf, int threads, size_t smem) {
  if (precision == EVORA_FP32) return f32::batch_max_ctas_per_sm(nf, threads, smem);
  return strict ? f64s::batch_max_ctas_per_sm(nf, threads, smem) : f64::batch_max_ctas_per_sm(nf, threads, smem);
}

namespace {

// Range of tubes [t0, t1) and its cells for tube index `tube` (-1 = all).
bool tube_range(const evora_batch* b, int tube, int* t0, int* t1, long long* off, long long* cells) {
  if (tube < -1 || tube >= b->ntubes) return false;
  if (tube == -1) {
    *t0 = 0;
    *t1 = b->ntubes;
    *off = 0;
    *cells = b->ntot;
  } else {
    *t0 = tube;
    *t1 = tube + 1;
    *off = b->offset[tube];
    *cells = b->n[tube];
  }
  return true;
}

int stage(evora_batch* b, size_t bytes) {
  if (b->aos_bytes >= bytes) return 0;
  cudaFree(b->aos_stage);
  b->aos_stage = nullptr;
  b->aos_bytes = 0;
  if (cudaMalloc(&b->aos_stage, bytes) != cudaSuccess) {
    cudaGetLastError();
    return EVORA_ERR_NOMEM;
  }
  b->aos_bytes = bytes;
  return 0;
}

void free_batch(evora_batch* b) {
  if (!b) return;
  drop_graphs(b);
  cudaFree(b->q);
  cudaFree(b->tubes);
  cudaFree(b->order);
  cudaFree(b->head);
  cudaFree(b->cell_updates);
  cudaFree(b->aos_stage);
  cudaFree(b->gscratch);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // namespace

extern "C" {

int evora_batch_create(const evora_params* p, int32_t ntubes, const int32_t* n, int32_t precision, int32_t flags,
                       evora_batch** out) {
  if (!p || !n || !out || ntubes < 1) return EVORA_ERR_ARG;
  if (precision != EVORA_FP32 && precision != EVORA_FP64) return EVORA_ERR_ARG;
  *out = nullptr;
  // the tubes run the hydro step alone: the substeps after it (gravity,
  // chemistry and floors, conduction, comoving terms) belong to resident grids
  if (p->gravity || p->chemistry || p->tempfloor || p->jeansfloor || p->conduction || p->supercomoving)
    return EVORA_ERR_ARG;
  int nmax = 0;
  long long ntot = 0;
  for (int i = 0; i < ntubes; ++i) {
    if (n[i] < 2) return EVORA_ERR_ARG;
    nmax = std::max(nmax, (int)n[i]);
    ntot += n[i];
  }
  evora_params pp = *p;
  pp.nx = nmax;
  pp.ny = pp.nz = 1;
  evora_batch* b = new (std::nothrow) evora_batch();
  if (!b) return EVORA_ERR_NOMEM;
  int rc = 0;
  if (!params_to_hydro(&pp, &b->P, nullptr, &rc)) {
    delete b;
    return rc;
  }
  if (p->dualenergy && precision == EVORA_FP32) {
    delete b;
    return EVORA_ERR_ARG;
  }
  b->params = pp;
  b->precision = precision;
  b->flags = flags;
  b->strict = (flags & EVORA_STRICT) != 0;
  b->nf = (flags & EVORA_CARRY_ENTROPY) || p->dualenergy ? 6 : 5;
  b->ntubes = ntubes;
  b->n.assign(n, n + ntubes);
  b->offset.resize(ntubes);
  b->work.resize(ntubes);
  b->tend.assign(ntubes, p->tend);
  long long off = 0;
  for (int i = 0; i < ntubes; ++i) {
    b->offset[i] = off;
    off += n[i];
    b->work[i] = (double)n[i] * (double)n[i];
  }
  b->ntot = ntot;
  b->nmax = nmax;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
  b->own_stream = true;
  if (cudaMalloc(&b->q, (size_t)b->nf * ntot * esize(b)) != cudaSuccess) goto fail;
  if (cudaMalloc(&b->tubes, sizeof(TubeState) * ntubes) != cudaSuccess) goto fail;
  if (cudaMalloc(&b->order, sizeof(int) * ntubes) != cudaSuccess) goto fail;
  if (cudaMalloc(&b->head, sizeof(int)) != cudaSuccess) goto fail;
  if (cudaMalloc(&b->cell_updates, sizeof(unsigned long long)) != cudaSuccess) goto fail;
  if (cudaMemset(b->cell_updates, 0, sizeof(unsigned long long)) != cudaSuccess) goto fail;
  {
    std::vector<TubeState> ts(ntubes);
    for (int i = 0; i < ntubes; ++i) {
      ts[i] = TubeState{};
      ts[i].offset = b->offset[i];
      ts[i].n = n[i];
      ts[i].status = TUBE_IDLE;
      ts[i].t = p->tstart;
      ts[i].tend = p->tend;
    }
    if (cudaMemcpy(b->tubes, ts.data(), sizeof(TubeState) * ntubes, cudaMemcpyHostToDevice) != cudaSuccess) goto fail;
  }
  rc = configure(b, 256, cap_for(b, 2));
  if (rc) {
    free_batch(b);
    return rc;
  }
  *out = b;
  return 0;
fail:
  cudaGetLastError();
  free_batch(b);
  return EVORA_ERR_NOMEM;
}

int evora_batch_destroy(evora_batch* b) {
  if (!b) return EVORA_ERR_ARG;
  cudaStreamSynchronize(b->stream);
  free_batch(b);
  return 0;
}

int evora_batch_set_stream(evora_batch* b, void* stream) {
  if (!b || !stream) return EVORA_ERR_ARG;
  cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->own_stream = false;
  b->stream = (cudaStream_t)stream;
  return 0;
}

int evora_batch_set_q(evora_batch* b, int32_t tube, const double* q) {
  if (!b || !q) return EVORA_ERR_ARG;
  int t0, t1;
  long long off, cells;
  if (!tube_range(b, tube, &t0, &t1, &off, &cells)) return EVORA_ERR_ARG;
  const size_t bytes = (size_t)cells * EVORA_NQ * sizeof(double);
  const double* src = q;
  if (!is_device_pointer(q)) {
    int rc = stage(b, bytes);
    if (rc) return rc;
    CU(cudaMemcpyAsync(b->aos_stage, q, bytes, cudaMemcpyHostToDevice, b->stream));
    src = b->aos_stage;
    // queue order: estimated work n * steps ~ n^2 * max(|u| + a) of the IC
    const double g = b->P.g, g1 = b->P.g1;
    for (int t = t0; t < t1; ++t) {
      const double* qt = q + (size_t)(b->offset[t] - off) * EVORA_NQ;
      double smax = 0.0;
      for (int i = 0; i < b->n[t]; ++i) {
        const double* c = qt + (size_t)i * EVORA_NQ;
        double u = c[1] / c[0];
        double pr = g1 * (c[4] - 0.5 * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) / c[0]);
        double s = std::fabs(u) + std::sqrt(std::max(0.0, g * pr / c[0]));
        smax = std::max(smax, s);
      }
      b->work[t] = (double)b->n[t] * (double)b->n[t] * std::max(smax, 1e-30) * (b->tend[t] - b->params.tstart);
    }
    b->order_dirty = true;
  }
  if (b->precision == EVORA_FP32)
    k_tube_from_aos<float><<<grid_of(cells), 256, 0, b->stream>>>(src, (float*)b->q, b->ntot, off, cells, b->nf);
  else
    k_tube_from_aos<double><<<grid_of(cells), 256, 0, b->stream>>>(src, (double*)b->q, b->ntot, off, cells, b->nf);
  std::vector<TubeState> ts(t1 - t0);
  for (int t = t0; t < t1; ++t) {
    TubeState& s = ts[t - t0];
    s = TubeState{};
    s.offset = b->offset[t];
    s.n = b->n[t];
    s.status = TUBE_RUNNING;
    s.t = b->params.tstart;
    s.tend = b->tend[t];
  }
  CU(cudaMemcpyAsync(b->tubes + t0, ts.data(), sizeof(TubeState) * ts.size(), cudaMemcpyHostToDevice, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  return 0;
}

int evora_batch_get_q(evora_batch* b, int32_t tube, double* q) {
  if (!b || !q) return EVORA_ERR_ARG;
  int t0, t1;
  long long off, cells;
  if (!tube_range(b, tube, &t0, &t1, &off, &cells)) return EVORA_ERR_ARG;
  const size_t bytes = (size_t)cells * EVORA_NQ * sizeof(double);
  const bool dev = is_device_pointer(q);
  double* dst = q;
  if (!dev) {
    int rc = stage(b, bytes);
    if (rc) return rc;
    dst = b->aos_stage;
  }
  if (b->precision == EVORA_FP32)
    k_tube_to_aos<float><<<grid_of(cells), 256, 0, b->stream>>>((const float*)b->q, dst, b->ntot, off, cells, b->nf,
                                                                  b->P.g1);
  else
    k_tube_to_aos<double><<<grid_of(cells), 256, 0, b->stream>>>((const double*)b->q, dst, b->ntot, off, cells,
                                                                   b->nf, b->P.g1);
  if (!dev) CU(cudaMemcpyAsync(q, dst, bytes, cudaMemcpyDeviceToHost, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  return 0;
}

int evora_batch_set_tend(evora_batch* b, int32_t tube, double tend) {
  if (!b || tube < 0 || tube >= b->ntubes) return EVORA_ERR_ARG;
  b->tend[tube] = tend;
  CU(cudaMemcpyAsync(&b->tubes[tube].tend, &b->tend[tube], sizeof(double), cudaMemcpyHostToDevice, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  return 0;
}

int evora_batch_run(evora_batch* b, int32_t max_steps, int32_t sync) {
  if (!b) return EVORA_ERR_ARG;
  if (b->order_dirty) {
    int rc = upload_order(b);
    if (rc) return rc;
  }
  // "to completion" is bounded too: at most 2^24 steps per tube per launch
  const int budget = max_steps <= 0 ? (1 << 24) : max_steps;
  auto it = b->graphs.find(budget);
  if (it == b->graphs.end()) {
    // capture: reset the queue head, then the persistent kernel
    b->plan.budget = budget;
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->head, 0, sizeof(int), b->stream);
    b->launch(b->plan, b->q, b->stream);
    CU(cudaStreamEndCapture(b->stream, &g));
    cudaGraphExec_t ex;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      set_cuda_error(e, "cudaGraphInstantiate");
      return EVORA_ERR_CUDA;
    }
    it = b->graphs.emplace(budget, ex).first;
  }
  CU(cudaGraphLaunch(it->second, b->stream));
  if (sync) {
    CU(cudaStreamSynchronize(b->stream));
    std::vector<TubeState> ts(b->ntubes);
    CU(cudaMemcpy(ts.data(), b->tubes, sizeof(TubeState) * ts.size(), cudaMemcpyDeviceToHost));
    unsigned e = 0;
    for (auto& s : ts) e |= s.err;
    return (int)e;
  }
  return 0;
}

int evora_batch_info(evora_batch* b, int32_t tube, double* t, double* dt, int32_t* go, int64_t* k, int32_t* status) {
  if (!b || tube < 0 || tube >= b->ntubes) return EVORA_ERR_ARG;
  TubeState s;
  CU(cudaMemcpyAsync(&s, b->tubes + tube, sizeof s, cudaMemcpyDeviceToHost, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  if (t) *t = s.t;
  if (dt) *dt = s.dt;
  if (go) *go = s.status == TUBE_RUNNING ? 1 : 0;
  if (k) *k = s.k;
  if (status) *status = s.status;
  return (int)s.err;
}

int evora_batch_steps_done(evora_batch* b, int64_t* cell_updates) {
  if (!b || !cell_updates) return EVORA_ERR_ARG;
  unsigned long long v = 0;
  CU(cudaMemcpyAsync(&v, b->cell_updates, sizeof v, cudaMemcpyDeviceToHost, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  *cell_updates = (int64_t)v;
  return 0;
}

int evora_batch_configure(evora_batch* b, int32_t threads, int32_t ctas_per_sm) {
  if (!b || (threads != 128 && threads != 256 && threads != 512) || ctas_per_sm < 1 || ctas_per_sm > 8)
    return EVORA_ERR_ARG;
  CU(cudaStreamSynchronize(b->stream));
  return configure(b, threads, cap_for(b, ctas_per_sm));
}

int evora_batch_autotune(evora_batch* b, int32_t steps, int32_t* threads_out, int32_t* ctas_out) {
  if (!b || steps < 1) return EVORA_ERR_ARG;
  if (b->order_dirty) {
    int rc = upload_order(b);
    if (rc) return rc;
  }
  // Save the state and the tube table, time each configuration for `steps`
  // steps per tube, restore after each trial.
  const size_t qbytes = (size_t)b->nf * b->ntot * esize(b);
  void* save_q = nullptr;
  TubeState* save_t = nullptr;
  if (cudaMalloc(&save_q, qbytes) != cudaSuccess || cudaMalloc(&save_t, sizeof(TubeState) * b->ntubes) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(save_q);
    return EVORA_ERR_NOMEM;
  }
  unsigned long long cu0 = 0;
  CU(cudaMemcpy(&cu0, b->cell_updates, sizeof cu0, cudaMemcpyDeviceToHost));
  CU(cudaMemcpyAsync(save_q, b->q, qbytes, cudaMemcpyDeviceToDevice, b->stream));
  CU(cudaMemcpyAsync(save_t, b->tubes, sizeof(TubeState) * b->ntubes, cudaMemcpyDeviceToDevice, b->stream));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  const int cand_threads[3] = {128, 256, 512};
  const int cand_ctas[3] = {1, 2, 3};
  float best = 1e30f;
  int bt = 256, bc = 2;
  for (int ti = 0; ti < 3; ++ti)
    for (int ci = 0; ci < 3; ++ci) {
      if (configure(b, cand_threads[ti], cap_for(b, cand_ctas[ci]))) continue;
      b->plan.budget = steps;
      CU(cudaEventRecord(e0, b->stream));
      cudaMemsetAsync(b->head, 0, sizeof(int), b->stream);
      b->launch(b->plan, b->q, b->stream);
      CU(cudaEventRecord(e1, b->stream));
      CU(cudaEventSynchronize(e1));
      CU(cudaGetLastError());
      float ms = 0.f;
      CU(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        bt = cand_threads[ti];
        bc = cand_ctas[ci];
      }
      CU(cudaMemcpyAsync(b->q, save_q, qbytes, cudaMemcpyDeviceToDevice, b->stream));
      CU(cudaMemcpyAsync(b->tubes, save_t, sizeof(TubeState) * b->ntubes, cudaMemcpyDeviceToDevice, b->stream));
    }
  CU(cudaMemcpyAsync(b->cell_updates, &cu0, sizeof cu0, cudaMemcpyHostToDevice, b->stream));
  CU(cudaStreamSynchronize(b->stream));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(save_q);
  cudaFree(save_t);
  if (threads_out) *threads_out = bt;
  if (ctas_out) *ctas_out = bc;
  return configure(b, bt, cap_for(b, bc));
}

}  // extern "C"
