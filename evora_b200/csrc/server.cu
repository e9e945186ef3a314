// server.cu -- a request loop for hydro solves with continuous batching
// (no counterpart in the reference, which runs one simulation per process).
//
// A request is an initial state q(6, nx, ny, nz) in the reference layout, a
// grid size and an end time.  The loop (evora_server_tick) admits pending
// requests in arrival order while their device footprint fits the HBM
// budget, keeps every admitted state resident, and on each tick advances all
// active work by up to `steps_per_tick` steps:
//   * 1D requests become tubes of one shared pool (a packed arena plus a tube
//     table) advanced together by one persistent launch of the batched-tube
//     kernel (batch_kernel.cuh), each tube with its own dt and t;
//   * 2D and 3D requests become resident grids (grid.cu) advanced together by
//     one multi-grid batch (evora_multigrid_*: per step one control kernel,
//     one persistent update launch over the tiles of all grids, one closing
//     kernel) on its own stream, concurrently with the tube launch; grids the
//     batch cannot take step on their own streams.
// Requests that arrive while others run are admitted at the next tick, as
// memory and tube slots free up.  Finished requests are read back and their
// time to solution (submit -> read back) is recorded.  A request's arithmetic
// does not depend on what else is in flight.
//
// Host copies: a request's state goes through a pool of page-locked buffers,
// copied there at submit, or, for evora_server_submit_borrowed, by the
// server's copy threads after submit (and the result likewise into the
// caller's array), so that those copies overlap the device's rounds.  The
// uploads, conversions and read-backs of a round are enqueued and waited for
// once per round.
//
// One host thread drives a server; the server's own worker threads only
// run host copies of request states (Stager).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/evora_gpu.h"
#include "batch.h"
#include "common.h"
#include "stager.h"

using namespace evora;

namespace {

using Clock = std::chrono::steady_clock;

// REQ_FINISHING: done on the device, result not yet read back;
// REQ_DELIVERING: read back, being copied into a borrowed array (both
// reported as running).
enum ReqState {
  REQ_PENDING = 0,
  REQ_RUNNING = 1,
  REQ_DONE = 2,
  REQ_FAILED = 3,
  REQ_FINISHING = 4,
  REQ_DELIVERING = 5
};

// A host buffer of doubles from the server's pool of page-locked buffers
// (so that uploads and read-backs are direct DMA), or pageable memory when
// page-locked memory could not be had.
struct HostBuf {
  double* p = nullptr;
  size_t cap = 0;      // doubles
  bool pinned = false;
};

struct Request {
  int64_t id = 0;
  int nx = 0, ny = 0, nz = 0;
  double tend = 0.0;
  int bt = 0;                    // boundary type (0: the server's)
  HostBuf q0;                    // initial state (host copy), released at admission
  double t_submit = 0.0, t_done = 0.0;
  int state = REQ_PENDING;
  bool tube = false;
  int slot = -1;                 // tube slot
  long long off = 0;             // arena offset (tubes)
  evora_grid* grid = nullptr;    // 2D/3D
  bool batched = false;          // stepped by the server's multi-grid batch
  bool uploading = false;        // admitted this round, its upload still in flight
  int stream = 0;                // index into the server's grid streams
  size_t bytes = 0;              // device footprint (grids)
  int64_t steps = 0;
  int round_steps = 1;           // steps per round (grids)
  unsigned err = 0;
  HostBuf result;                // read back state, released when delivered
  size_t result_n = 0;
  // evora_server_submit_borrowed: the caller's arrays, and the chunks of the
  // copy in flight (the initial state into q0, then the result into out)
  const double* src = nullptr;
  double* out = nullptr;
  std::unique_ptr<std::atomic<int>> left;
  long long cells() const { return (long long)nx * ny * nz; }
};

#define CU(call)                 \
  do {                           \
    cudaError_t e_ = (call);     \
    if (e_ != cudaSuccess) {     \
      set_cuda_error(e_, #call); \
      return EVORA_ERR_CUDA;     \
    }                            \
  } while (0)

}  // namespace

struct evora_server {
  evora_params base{};
  HydroParams P{};
  int precision = EVORA_FP32;
  int flags = 0;
  int nf = 5;
  size_t budget = 0, used = 0;
  int steps_per_tick = 64;       // base step count of a round
  int max_round_steps = 512;     // cap on a grid's / the tube launch's steps per round
  Clock::time_point t0;
  int64_t next_id = 1;
  std::deque<int64_t> pending;
  std::map<int64_t, Request> reqs;
  // tube pool
  int max_slots = 0;
  int max_tube = 0;
  long long arena = 0;
  void* q = nullptr;
  TubeState* tubes = nullptr;
  int* order = nullptr;
  int* head = nullptr;
  unsigned long long* cu = nullptr;
  void* gscratch = nullptr;
  // AoS staging of tubes (stage: the round's admissions, stage2: read-backs
  // in flight), stage_cells cells each; the tubes' copies and conversions
  // are enqueued on the read-back stream and waited for once per round
  double* stage = nullptr;
  double* stage2 = nullptr;
  long long stage_cells = 0, stage_used = 0, stage2_used = 0;
  std::vector<Request*> tube_uploads;  // tubes admitted this round
  std::vector<Request*> tube_reads;    // tubes whose read-backs are in flight
  std::deque<Request*> tube_waiting;   // finished tubes waiting for room in stage2
  std::vector<TubeState> ts_host;      // host sources of the tube-table uploads, by slot
  cudaStream_t rstream = nullptr;  // read-back of finished tubes
  std::vector<int> free_streams;   // indices of idle grid streams
  std::vector<Request*> to_free;   // grids read back, destroyed after the round
  std::vector<Request*> uploads;   // grids admitted this round (uploads in flight)
  std::vector<Request*> delivering;  // results being copied into borrowed arrays
  std::deque<int64_t> completed;   // ids finished since the last evora_server_completed
  std::vector<int64_t> slot_req; // slot -> request id (0 = free)
  std::vector<std::pair<long long, long long>> free_seg;  // (offset, length), sorted
  BatchPlan plan{};
  BatchLaunch launch = nullptr;
  bool order_dirty = true;
  int active_tubes = 0;
  cudaStream_t tstream = nullptr;
  cudaStream_t mstream = nullptr;  // the multi-grid batch
  evora_multigrid* mg = nullptr;
  int batched_grids = 0;
  std::vector<cudaStream_t> gstreams;
  int next_stream = 0;
  std::vector<double> latencies;
  long long grid_cell_updates = 0;
  double first_submit = -1.0, last_done = 0.0;
  size_t fixed = 0;              // arena and staging
  // page-locked host buffers by size class (powers of two of doubles)
  std::map<int, std::vector<HostBuf>> free_bufs;
  Stager copies;
  // host time per round phase: launch, read-back, admission, wait, free, detect
  double phase_s[6] = {0, 0, 0, 0, 0, 0};
  // device time of the rounds' tube launches and multi-grid steps (events
  // around them on their streams), ms
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double dev_ms[2] = {0.0, 0.0};
  long long rounds = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  size_t esize() const { return precision == EVORA_FP32 ? 4 : 8; }
};

namespace {

HostBuf buf_get(evora_server* s, size_t n) {
  int cls = 10;
  while (((size_t)1 << cls) < n) ++cls;
  // the smallest free buffer of this size class or a larger one (pinning new
  // memory costs far more than holding a larger buffer for a while)
  for (auto it = s->free_bufs.lower_bound(cls); it != s->free_bufs.end(); ++it) {
    if (it->second.empty()) continue;
    HostBuf b = it->second.back();
    it->second.pop_back();
    return b;
  }
  HostBuf b;
  b.cap = (size_t)1 << cls;
  if (cudaHostAlloc((void**)&b.p, b.cap * sizeof(double), cudaHostAllocDefault) == cudaSuccess) {
    b.pinned = true;
  } else {
    cudaGetLastError();
    b.p = static_cast<double*>(std::malloc(b.cap * sizeof(double)));
    b.pinned = false;
  }
  if (!b.p) b.cap = 0;
  return b;
}

void buf_put(evora_server* s, HostBuf& b) {
  if (!b.p) return;
  int cls = 10;
  while (((size_t)1 << cls) < b.cap) ++cls;
  s->free_bufs[cls].push_back(b);
  b = HostBuf{};
}

void buf_free(HostBuf& b) {
  if (!b.p) return;
  if (b.pinned) cudaFreeHost(b.p);
  else std::free(b.p);
  b = HostBuf{};
}

bool alloc_segment(evora_server* s, long long n, long long* off) {
  for (size_t i = 0; i < s->free_seg.size(); ++i) {
    auto& seg = s->free_seg[i];
    if (seg.second >= n) {
      *off = seg.first;
      seg.first += n;
      seg.second -= n;
      if (seg.second == 0) s->free_seg.erase(s->free_seg.begin() + (long)i);
      return true;
    }
  }
  return false;
}

void free_segment(evora_server* s, long long off, long long n) {
  auto& fs = s->free_seg;
  auto it = std::lower_bound(fs.begin(), fs.end(), std::make_pair(off, 0LL));
  it = fs.insert(it, {off, n});
  // merge with neighbours
  size_t i = (size_t)(it - fs.begin());
  if (i + 1 < fs.size() && fs[i].first + fs[i].second == fs[i + 1].first) {
    fs[i].second += fs[i + 1].second;
    fs.erase(fs.begin() + (long)i + 1);
  }
  if (i > 0 && fs[i - 1].first + fs[i - 1].second == fs[i].first) {
    fs[i - 1].second += fs[i].second;
    fs.erase(fs.begin() + (long)i);
  }
}

size_t grid_bytes(const evora_server* s, long long cells) {
  // two SoA copies + the reference-layout staging used by set_q / get_q
  return (size_t)cells * (2 * (size_t)s->nf * s->esize() + EVORA_NQ * sizeof(double)) + (1 << 16);
}

int admit(evora_server* s, Request& r) {
  if (r.tube) {
    if (s->stage_used + r.nx > s->stage_cells) return 1;   // the round's staging is full: next round
    int slot = -1;
    for (int i = 0; i < s->max_slots; ++i)
      if (s->slot_req[i] == 0) {
        slot = i;
        break;
      }
    long long off = 0;
    if (slot < 0 || !alloc_segment(s, r.nx, &off)) return 1;   // not now
    r.slot = slot;
    r.off = off;
    s->slot_req[slot] = r.id;
    // enqueued on the read-back stream (the running tube launch never
    // touches a free slot or a free arena segment); waited for, and the host
    // copy released, after the round (join_tube_uploads)
    double* st = s->stage + (size_t)EVORA_NQ * s->stage_used;
    CU(cudaMemcpyAsync(st, r.q0.p, sizeof(double) * EVORA_NQ * r.nx, cudaMemcpyHostToDevice, s->rstream));
    tube_from_aos(st, s->q, s->precision == EVORA_FP32, s->arena, off, r.nx, s->nf, s->rstream);
    TubeState& ts = s->ts_host[slot];
    ts = TubeState{};
    ts.offset = off;
    ts.n = r.nx;
    ts.status = TUBE_RUNNING;
    ts.t = s->base.tstart;
    ts.tend = r.tend;
    ts.bt = r.bt;
    CU(cudaMemcpyAsync(s->tubes + slot, &ts, sizeof ts, cudaMemcpyHostToDevice, s->rstream));
    s->stage_used += r.nx;
    s->tube_uploads.push_back(&r);
    s->active_tubes++;
    s->order_dirty = true;
  } else {
    const size_t bytes = grid_bytes(s, r.cells());
    if (s->used + bytes > s->budget) return 1;
    evora_params p = s->base;
    p.nx = r.nx;
    p.ny = r.ny;
    p.nz = r.nz;
    p.tend = r.tend;
    if (r.bt) p.boundtype = r.bt;
    evora_grid* g = nullptr;
    // a stream per running grid (recycled), so that waiting for or reading
    // back one grid never waits for another; the grid's memory is
    // stream-ordered on it, so retiring a grid never synchronises the device
    if (s->free_streams.empty()) {
      cudaStream_t st;
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return 1;
      }
      s->gstreams.push_back(st);
      s->free_streams.push_back((int)s->gstreams.size() - 1);
    }
    const int si = s->free_streams.back();
    int rc = evora_grid_create_async(&p, s->precision, s->flags & ~EVORA_REFERENCE_KERNELS, s->gstreams[si], &g);
    if (rc) return rc == EVORA_ERR_NOMEM ? 1 : rc;
    s->free_streams.pop_back();
    r.stream = si;
    // enqueued only: the upload and conversion run on the grid's stream
    // while the host admits the next requests; the grid joins the batch
    // once the round's wait has seen them complete (join_uploads)
    rc = grid_set_q_async(g, r.q0.p);
    if (rc) {
      cudaStreamSynchronize(s->gstreams[si]);
      evora_grid_destroy(g);
      s->free_streams.push_back(si);
      return rc == EVORA_ERR_NOMEM ? 1 : rc;
    }
    r.grid = g;
    r.bytes = bytes;
    r.uploading = true;
    s->uploads.push_back(&r);
    // time quantum: a round gives each grid about the same device time, so
    // its step count falls with its size (2^20 cell-updates per base step)
    const double quantum = (double)s->steps_per_tick * (double)(1 << 20);
    r.round_steps = (int)std::max(1.0, std::min((double)s->max_round_steps, quantum / (double)r.cells()));
    s->used += bytes;
  }
  r.state = REQ_RUNNING;
  return 0;
}

// Tubes admitted this round: their uploads are complete once the read-back
// stream is; their host copies go back to the pool.
int join_tube_uploads(evora_server* s) {
  if (s->tube_uploads.empty()) return 0;
  CU(cudaStreamSynchronize(s->rstream));
  for (Request* r : s->tube_uploads) buf_put(s, r->q0);
  s->tube_uploads.clear();
  s->stage_used = 0;
  return 0;
}

// Finished tubes: conversion to the reference layout into stage2 and the
// copy into a page-locked buffer, enqueued while the device is idle between
// rounds (as many as stage2 holds) and collected in the next round.
int issue_tube_reads(evora_server* s) {
  while (!s->tube_waiting.empty()) {
    Request& r = *s->tube_waiting.front();
    if (s->stage2_used + r.nx > s->stage_cells) break;
    r.result_n = (size_t)EVORA_NQ * r.cells();
    r.result = buf_get(s, r.result_n);
    if (!r.result.p) return EVORA_ERR_NOMEM;
    double* st = s->stage2 + (size_t)EVORA_NQ * s->stage2_used;
    tube_to_aos(s->q, st, s->precision == EVORA_FP32, s->arena, r.off, r.nx, s->nf, s->P.g1, s->rstream);
    CU(cudaMemcpyAsync(r.result.p, st, sizeof(double) * r.result_n, cudaMemcpyDeviceToHost, s->rstream));
    s->stage2_used += r.nx;
    s->tube_reads.push_back(&r);
    s->tube_waiting.pop_front();
  }
  return 0;
}

void finish(evora_server* s, Request& r, unsigned err) {
  r.err = err;
  r.state = err ? REQ_FAILED : REQ_DONE;
  r.t_done = s->now();
  s->last_done = r.t_done;
  s->latencies.push_back(r.t_done - r.t_submit);
  s->completed.push_back(r.id);
}

// Grids admitted this round: their uploads are complete once their streams
// are; the host copies go back to the pool and the grids join the batch
// (or step alone on their streams from the next round).
int join_uploads(evora_server* s) {
  for (Request* r : s->uploads) {
    CU(cudaStreamSynchronize(s->gstreams[r->stream]));
    buf_put(s, r->q0);
    r->uploading = false;
    r->batched = s->mg && evora_multigrid_add(s->mg, r->grid) == 0;
    if (r->batched) s->batched_grids++;
  }
  s->uploads.clear();
  return 0;
}

// A grid that finished: its read-back (conversion to the reference layout
// and the copy into a page-locked buffer) is enqueued on its stream at once
// and collected in the next round.
int start_readback(evora_server* s, Request& r) {
  r.result_n = (size_t)EVORA_NQ * r.cells();
  r.result = buf_get(s, r.result_n);
  if (!r.result.p) return EVORA_ERR_NOMEM;
  return grid_get_q_async(r.grid, r.result.p);
}

// A request's initial state: copied into the page-locked pool before
// returning, or (borrowed) by the copy threads after it, the request
// admissible once that copy is complete.
int submit(evora_server* s, int32_t nx, int32_t ny, int32_t nz, double tend, int32_t boundtype, const double* q0,
           double* q_out, bool borrowed, int64_t* id) {
  if (!s || !q0 || !id || nx < 2 || ny < 1 || nz < 1 || (nz > 1 && ny == 1)) return EVORA_ERR_ARG;
  if (boundtype < 0 || boundtype > 3) return EVORA_ERR_ARG;
  const bool tube = (ny == 1 && nz == 1);
  if (tube && nx > s->max_tube) return EVORA_ERR_ARG;
  Request r;
  r.nx = nx;
  r.ny = ny;
  r.nz = nz;
  if (!tube && grid_bytes(s, r.cells()) > s->budget - s->fixed) return EVORA_ERR_ARG;   // could never fit
  r.id = s->next_id++;
  r.tend = tend;
  r.bt = boundtype;
  r.tube = tube;
  const size_t nq = (size_t)EVORA_NQ * nx * ny * nz;
  // the page-locked buffer is taken here, on the driving thread: pinning new
  // memory on a copy thread was measured to stall this thread's CUDA calls
  // for longer than the pinning itself
  r.q0 = buf_get(s, nq);
  if (!r.q0.p) return EVORA_ERR_NOMEM;
  if (borrowed) {
    r.src = q0;
    r.out = q_out;
    r.left.reset(new (std::nothrow) std::atomic<int>(0));
    if (!r.left) {
      buf_put(s, r.q0);
      return EVORA_ERR_NOMEM;
    }
    s->copies.post(r.q0.p, q0, nq * sizeof(double), r.left.get());
  } else {
    s->copies.copy(r.q0.p, q0, nq * sizeof(double));
  }
  r.t_submit = s->now();
  if (s->first_submit < 0) s->first_submit = r.t_submit;
  *id = r.id;
  s->pending.push_back(r.id);
  s->reqs.emplace(r.id, std::move(r));
  return 0;
}

// A result read back into the page-locked pool: delivered now, or first
// copied into the caller's borrowed array by the copy threads.
void deliver(evora_server* s, Request& r, unsigned err) {
  if (r.out && r.result.p) {
    r.err = err;
    r.state = REQ_DELIVERING;
    s->copies.post(r.out, r.result.p, sizeof(double) * r.result_n, r.left.get());
    s->delivering.push_back(&r);
    return;
  }
  finish(s, r, err);
}

// Results whose copies into borrowed arrays are complete are finished.
void collect_deliveries(evora_server* s) {
  size_t k = 0;
  for (Request* r : s->delivering) {
    if (r->left->load(std::memory_order_acquire) > 0) {
      s->delivering[k++] = r;
      continue;
    }
    buf_put(s, r->result);
    finish(s, *r, r->err);
  }
  s->delivering.resize(k);
}

int upload_order(evora_server* s) {
  std::vector<int> ord;
  std::vector<double> work;
  for (int i = 0; i < s->max_slots; ++i)
    if (s->slot_req[i]) {
      const Request& r = s->reqs[s->slot_req[i]];
      if (r.state != REQ_RUNNING) continue;
      ord.push_back(i);
    }
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    return s->reqs[s->slot_req[a]].nx > s->reqs[s->slot_req[b]].nx;
  });
  if (!ord.empty())
    CU(cudaMemcpyAsync(s->order, ord.data(), sizeof(int) * ord.size(), cudaMemcpyHostToDevice, s->tstream));
  s->plan.ntubes = (int)ord.size();
  s->order_dirty = false;
  return 0;
}

}  // namespace

extern "C" {

int evora_server_create(const evora_params* base, int32_t precision, int32_t flags, double hbm_budget_bytes,
                        int32_t steps_per_tick, int32_t max_tube_cells, int32_t max_tubes, evora_server** out) {
  if (!base || !out || hbm_budget_bytes <= 0 || steps_per_tick < 1 || max_tube_cells < 2 || max_tubes < 1)
    return EVORA_ERR_ARG;
  if (precision != EVORA_FP32 && precision != EVORA_FP64) return EVORA_ERR_ARG;
  *out = nullptr;
  evora_server* s = new (std::nothrow) evora_server();
  if (!s) return EVORA_ERR_NOMEM;
  s->base = *base;
  s->precision = precision;
  s->flags = flags;
  s->nf = (flags & EVORA_CARRY_ENTROPY) || base->dualenergy ? 6 : 5;
  s->budget = (size_t)hbm_budget_bytes;
  s->steps_per_tick = steps_per_tick;
  s->t0 = Clock::now();
  s->max_slots = max_tubes;
  s->max_tube = max_tube_cells;
  evora_params pp = *base;
  pp.nx = max_tube_cells;
  pp.ny = pp.nz = 1;
  int rc = 0;
  if (!params_to_hydro(&pp, &s->P, nullptr, &rc)) {
    delete s;
    return rc;
  }
  // the tube arena takes a quarter of the budget, at least one tube per slot of average size
  s->arena = std::max<long long>((long long)max_tube_cells,
                                 (long long)(s->budget / 4 / ((size_t)s->nf * s->esize())));
  const size_t arena_bytes = (size_t)s->arena * s->nf * s->esize();
  s->slot_req.assign(max_tubes, 0);
  s->free_seg = {{0, s->arena}};
  if (cudaStreamCreateWithFlags(&s->tstream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
  {
    // keep memory freed by retired grids in the device's default pool for
    // the next admissions instead of returning it to the driver
    int dev = 0;
    cudaMemPool_t pool;
    cudaGetDevice(&dev);
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = (uint64_t)s->budget;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  if (cudaStreamCreateWithFlags(&s->rstream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
  for (auto& e : s->ev)
    if (cudaEventCreate(&e) != cudaSuccess) goto fail;
  if (cudaStreamCreateWithFlags(&s->mstream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
  if (evora_multigrid_create(precision, flags & ~EVORA_REFERENCE_KERNELS, s->mstream, &s->mg)) s->mg = nullptr;
  // tube staging: up to 64 tubes of the largest size per round, within a
  // sixteenth of the budget
  s->stage_cells = std::max<long long>(max_tube_cells,
                                       std::min<long long>(64LL * max_tube_cells,
                                                           (long long)(s->budget / 16 / (EVORA_NQ * sizeof(double)))));
  s->ts_host.assign(max_tubes, TubeState{});
  if (cudaMalloc(&s->stage2, sizeof(double) * EVORA_NQ * s->stage_cells) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->q, arena_bytes) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->tubes, sizeof(TubeState) * max_tubes) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->order, sizeof(int) * max_tubes) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->head, sizeof(int)) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->cu, sizeof(unsigned long long)) != cudaSuccess) goto fail;
  if (cudaMemset(s->cu, 0, sizeof(unsigned long long)) != cudaSuccess) goto fail;
  if (cudaMalloc(&s->stage, sizeof(double) * EVORA_NQ * s->stage_cells) != cudaSuccess) goto fail;
  {
    std::vector<TubeState> ts(max_tubes);
    for (auto& t : ts) {
      t = TubeState{};
      t.status = TUBE_IDLE;
    }
    if (cudaMemcpy(s->tubes, ts.data(), sizeof(TubeState) * max_tubes, cudaMemcpyHostToDevice) != cudaSuccess)
      goto fail;
  }
  {
    BatchPlan& pl = s->plan;
    pl.P = s->P;
    pl.xmin = base->xmin;
    pl.xmax = base->xmax;
    pl.nf = s->nf;
    pl.ntot = s->arena;
    pl.tubes = s->tubes;
    pl.order = s->order;
    pl.ntubes = 0;
    pl.head = s->head;
    // a round gives each tube about steps_per_tick * 2^14 cell-steps (at
    // most 8 * steps_per_tick steps), so long and short tubes take similar
    // device time per round
    s->max_round_steps = 8 * steps_per_tick;
    pl.budget = 8 * steps_per_tick;
    pl.quantum = (long long)steps_per_tick << 14;
    pl.nmax = max_tube_cells;
    pl.cell_updates = s->cu;
    const size_t per_cell = (size_t)(s->nf + 5) * s->esize();
    // one CTA of 512 threads per SM, the largest shared-memory staging
    pl.cap = std::min(max_tube_cells, (int)((227 * 1024 - 4096) / per_cell) - 4);
    s->launch = batch_pick_for(precision, (flags & EVORA_STRICT) != 0, s->nf, 512, &pl);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = batch_ctas_per_sm(precision, (flags & EVORA_STRICT) != 0, s->nf, 512, pl.smem);
    pl.ctas = std::max(1, sms * std::max(1, per_sm));
    if (max_tube_cells > pl.cap) {
      size_t need = (size_t)pl.ctas * (size_t)(s->nf + 5) * (size_t)(max_tube_cells + 4) * s->esize();
      if (cudaMalloc(&s->gscratch, need) != cudaSuccess) goto fail;
    }
    pl.gscratch = s->gscratch;
  }
  s->used = arena_bytes + 2 * sizeof(double) * EVORA_NQ * (size_t)s->stage_cells;
  s->fixed = s->used;
  if (s->used > s->budget) {
    evora_server_destroy(s);
    return EVORA_ERR_ARG;
  }
  *out = s;
  return 0;
fail:
  cudaGetLastError();
  evora_server_destroy(s);
  return EVORA_ERR_NOMEM;
}

int evora_server_destroy(evora_server* s) {
  if (!s) return EVORA_ERR_ARG;
  s->copies.stop();   // no copy into a buffer freed below is still queued
  cudaDeviceSynchronize();
  if (s->mg) evora_multigrid_destroy(s->mg);
  for (auto& kv : s->reqs) {
    if (kv.second.grid) evora_grid_destroy(kv.second.grid);
    buf_free(kv.second.q0);
    buf_free(kv.second.result);
  }
  for (auto& kv : s->free_bufs)
    for (auto& b : kv.second) buf_free(b);
  cudaFree(s->q);
  cudaFree(s->tubes);
  cudaFree(s->order);
  cudaFree(s->head);
  cudaFree(s->cu);
  cudaFree(s->gscratch);
  cudaFree(s->stage);
  cudaFree(s->stage2);
  if (s->rstream) cudaStreamDestroy(s->rstream);
  for (auto e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->tstream) cudaStreamDestroy(s->tstream);
  if (s->mstream) cudaStreamDestroy(s->mstream);
  for (auto st : s->gstreams) cudaStreamDestroy(st);
  delete s;
  return 0;
}

int evora_server_submit(evora_server* s, int32_t nx, int32_t ny, int32_t nz, double tend, int32_t boundtype,
                        const double* q0, int64_t* id) {
  return submit(s, nx, ny, nz, tend, boundtype, q0, nullptr, false, id);
}

int evora_server_submit_borrowed(evora_server* s, int32_t nx, int32_t ny, int32_t nz, double tend,
                                 int32_t boundtype, const double* q0, double* q_out, int64_t* id) {
  return submit(s, nx, ny, nz, tend, boundtype, q0, q_out, true, id);
}

int evora_server_tick(evora_server* s, int32_t* n_active, int32_t* n_pending) {
  if (!s) return EVORA_ERR_ARG;
  double tp = s->now();
  auto mark = [&](int phase) {
    const double t = s->now();
    s->phase_s[phase] += t - tp;
    tp = t;
  };
  // 1. (admission happens below, while the round runs; new work starts next round)
  // 2. launch one round of steps for everything running: the tube launch and
  //    each grid's graph on its own stream, concurrently
  if (s->order_dirty) {
    int rc = upload_order(s);
    if (rc) return rc;
  }
  const bool timed_tubes = s->plan.ntubes > 0 && s->ev[0];
  if (s->plan.ntubes > 0) {
    if (timed_tubes) CU(cudaEventRecord(s->ev[0], s->tstream));
    CU(cudaMemsetAsync(s->head, 0, sizeof(int), s->tstream));
    s->launch(s->plan, s->q, s->tstream);
    CU(cudaGetLastError());
    if (timed_tubes) CU(cudaEventRecord(s->ev[1], s->tstream));
  }
  std::vector<Request*> grids;
  for (auto& kv : s->reqs)
    if (kv.second.state == REQ_RUNNING && kv.second.grid) {
      grids.push_back(&kv.second);
      if (kv.second.batched) continue;
      int rc = evora_grid_step(kv.second.grid, kv.second.round_steps, 0);
      if (rc) return rc;
    }
  const bool timed_batch = s->batched_grids > 0 && s->ev[2];
  if (s->batched_grids > 0) {
    if (timed_batch) CU(cudaEventRecord(s->ev[2], s->mstream));
    int rc = evora_multigrid_step(s->mg, s->steps_per_tick, 0);
    if (rc) return rc;
    if (timed_batch) CU(cudaEventRecord(s->ev[3], s->mstream));
  }
  mark(0);
  // 3. while the GPU works: collect the read-backs of what finished in the
  //    previous round (enqueued when it was detected)
  collect_deliveries(s);
  if (!s->tube_reads.empty()) {
    CU(cudaStreamSynchronize(s->rstream));
    for (Request* r : s->tube_reads) {
      free_segment(s, r->off, r->nx);
      s->slot_req[r->slot] = 0;
      deliver(s, *r, r->err);
    }
    s->tube_reads.clear();
    s->stage2_used = 0;
  }
  for (auto& kv : s->reqs) {
    Request& r = kv.second;
    if (r.state != REQ_FINISHING || r.tube) continue;
    CU(cudaStreamSynchronize(s->gstreams[r.stream]));
    s->grid_cell_updates += (long long)r.steps * r.cells();
    s->to_free.push_back(&r);
    deliver(s, r, r.err);
  }
  mark(1);
  // 3b. admission, in arrival order, while memory and slots allow (host
  //     copies overlap the round); admitted work starts with the next round
  while (!s->pending.empty()) {
    Request& r = s->reqs[s->pending.front()];
    if (r.left && r.left->load(std::memory_order_acquire) > 0) break;   // its state is still being copied
    int rc = admit(s, r);
    if (rc == 1) {
      bool idle = s->active_tubes == 0 && s->to_free.empty() && grids.empty();
      for (auto& kv : s->reqs)
        idle = idle && kv.second.state != REQ_RUNNING && kv.second.state != REQ_FINISHING &&
               kv.second.state != REQ_DELIVERING;
      if (!idle) break;           // head of the queue waits for room
      rc = EVORA_ERR_NOMEM;       // nothing running and still no room: it never fits
    }
    s->pending.pop_front();
    if (rc) finish(s, r, (unsigned)rc);
  }
  mark(2);
  // 4. wait for the round
  CU(cudaStreamSynchronize(s->tstream));
  CU(cudaStreamSynchronize(s->mstream));
  for (Request* r : grids)
    if (!r->batched) CU(cudaStreamSynchronize(s->gstreams[r->stream]));
  {
    float ms = 0.f;
    if (timed_tubes && cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]) == cudaSuccess) s->dev_ms[0] += ms;
    if (timed_batch && cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]) == cudaSuccess) s->dev_ms[1] += ms;
    cudaGetLastError();
  }
  {
    int rc = join_tube_uploads(s);
    if (rc) return rc;
  }
  mark(3);
  // 5. grids read back above can go now (their streams are idle)
  for (Request* r : s->to_free) {
    evora_grid_destroy(r->grid);
    r->grid = nullptr;
    s->used -= r->bytes;
    s->free_streams.push_back(r->stream);
  }
  s->to_free.clear();
  mark(4);
  // 6. detect finished work; it is read back during the next round
  if (s->plan.ntubes > 0) {
    std::vector<TubeState> ts(s->max_slots);
    CU(cudaMemcpy(ts.data(), s->tubes, sizeof(TubeState) * s->max_slots, cudaMemcpyDeviceToHost));
    for (int i = 0; i < s->max_slots; ++i) {
      if (!s->slot_req[i]) continue;
      Request& r = s->reqs[s->slot_req[i]];
      if (r.state != REQ_RUNNING || ts[i].status == TUBE_RUNNING) continue;
      r.steps = ts[i].k;
      r.err = ts[i].err;
      r.state = REQ_FINISHING;
      s->tube_waiting.push_back(&r);
      s->active_tubes--;
      s->order_dirty = true;
    }
  }
  {
    int rc = issue_tube_reads(s);
    if (rc) return rc;
  }
  if (s->batched_grids > 0) {
    // one read of the batch's status words; finished grids leave the batch
    // and are read back on their own streams during the next round
    const int nb = s->batched_grids;
    std::vector<evora_grid*> gs(nb);
    std::vector<int32_t> go(nb);
    std::vector<uint32_t> er(nb);
    std::vector<int64_t> kk(nb);
    int32_t n = 0;
    int rc = evora_multigrid_status(s->mg, gs.data(), go.data(), er.data(), kk.data(), nb, &n);
    if (rc) return rc;
    std::map<evora_grid*, int> done;
    for (int i = 0; i < n; ++i)
      if (!go[i] || er[i]) done[gs[i]] = i;
    for (Request* r : grids) {
      if (!r->batched) continue;
      auto it = done.find(r->grid);
      if (it == done.end()) continue;
      r->steps = kk[it->second];
      r->err = er[it->second];
      r->state = REQ_FINISHING;
      evora_multigrid_remove(s->mg, r->grid);
      r->batched = false;
      s->batched_grids--;
      int rc2 = start_readback(s, *r);
      if (rc2) return rc2;
    }
  }
  for (Request* r : grids) {
    if (r->batched || r->state != REQ_RUNNING) continue;
    double t, dt;
    int32_t go;
    int64_t k;
    int rc = evora_grid_time(r->grid, &t, &dt, &go, &k);
    if (rc) return rc;
    const int st = evora_grid_status(r->grid);
    if (go && !st) continue;
    r->steps = k;
    r->err = (unsigned)st;
    r->state = REQ_FINISHING;
    rc = start_readback(s, *r);
    if (rc) return rc;
  }
  // grids admitted this round join the batch after its status was read (a
  // batch changed since its last step reads each member's control block)
  {
    int rc = join_uploads(s);
    if (rc) return rc;
  }
  collect_deliveries(s);
  mark(5);
  s->rounds++;
  int act = 0;
  for (auto& kv : s->reqs)
    act += kv.second.state == REQ_RUNNING || kv.second.state == REQ_FINISHING || kv.second.state == REQ_DELIVERING;
  if (n_active) *n_active = act;
  if (n_pending) *n_pending = (int32_t)s->pending.size();
  return 0;
}

int evora_server_result(evora_server* s, int64_t id, double* q_out, double* latency_s, int64_t* steps,
                        int32_t* state) {
  if (!s) return EVORA_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    if (state) *state = -1;
    return EVORA_ERR_ARG;
  }
  Request& r = it->second;
  if (state) *state = r.state == REQ_FINISHING || r.state == REQ_DELIVERING ? REQ_RUNNING : r.state;
  if (r.state != REQ_DONE && r.state != REQ_FAILED) return 0;
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  if (steps) *steps = r.steps;
  if (q_out && r.result.p) s->copies.copy(q_out, r.result.p, sizeof(double) * r.result_n);
  else if (q_out && r.out && q_out != r.out && r.result_n)   // delivered into the borrowed array
    s->copies.copy(q_out, r.out, sizeof(double) * r.result_n);
  const int err = (int)r.err;
  if (q_out) {   // delivered
    buf_put(s, r.result);
    s->reqs.erase(it);
  }
  return err;
}

int evora_server_profile(evora_server* s, double out[7]) {
  if (!s || !out) return EVORA_ERR_ARG;
  for (int i = 0; i < 6; ++i) out[i] = s->phase_s[i];
  out[6] = (double)s->rounds;
  return 0;
}

int evora_server_device_ms(evora_server* s, double* tube_ms, double* batch_ms) {
  if (!s) return EVORA_ERR_ARG;
  if (tube_ms) *tube_ms = s->dev_ms[0];
  if (batch_ms) *batch_ms = s->dev_ms[1];
  return 0;
}

int evora_server_completed(evora_server* s, int64_t* ids, int32_t max_ids, int32_t* n) {
  if (!s || !n || (max_ids > 0 && !ids)) return EVORA_ERR_ARG;
  int32_t k = 0;
  while (k < max_ids && !s->completed.empty()) {
    ids[k++] = s->completed.front();
    s->completed.pop_front();
  }
  *n = k;
  return 0;
}

int evora_server_stats(evora_server* s, double* p50_s, double* p99_s, int64_t* completed, int64_t* cell_updates,
                       double* span_s) {
  if (!s) return EVORA_ERR_ARG;
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double f) {
    if (l.empty()) return 0.0;
    size_t i = (size_t)std::min<double>((double)l.size() - 1, std::ceil(f * l.size()) - 1);
    return l[i];
  };
  if (p50_s) *p50_s = pct(0.50);
  if (p99_s) *p99_s = pct(0.99);
  if (completed) *completed = (int64_t)l.size();
  if (cell_updates) {
    unsigned long long v = 0;
    CU(cudaMemcpy(&v, s->cu, sizeof v, cudaMemcpyDeviceToHost));
    *cell_updates = (int64_t)v + s->grid_cell_updates;
  }
  if (span_s) *span_s = s->first_submit < 0 ? 0.0 : s->last_done - s->first_submit;
  return 0;
}

}  // extern "C"
