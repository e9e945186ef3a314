// batch.h -- structures shared by the batched-tube kernel and its host code.
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

enum TubeStatus { TUBE_RUNNING = 0, TUBE_DONE = 1, TUBE_ERROR = 2, TUBE_IDLE = 3 };

// One tube's bookkeeping (device array, one entry per tube).
struct TubeState {
  long long offset;   // first cell of the tube in the packed state
  int n;              // cells
  int status;         // TubeStatus
  double t, dt, tend;
  long long k;        // steps done
  unsigned err;       // EVORA_ERR_* mask
  int bt;             // boundary type of this tube (0: the batch's)
};

template <typename T>
struct BatchArgs {
  HydroParams P;          // shared options (nx and dx are per tube)
  double xmin, xmax;
  T* q;                   // NF planes of ntot cells (tubes packed)
  long long ntot;
  TubeState* tubes;
  const int* order;       // queue order (tube indices, largest work first)
  int ntubes;
  int* head;              // queue head (reset to 0 before each launch)
  int budget;             // max steps per tube in this launch
  long long quantum;      // if > 0: a tube of n cells runs at most max(1, quantum / n) steps
  int cap;                // tubes with n <= cap live in shared memory
  int capw;               // cap < n <= capw: w in shared memory, q in the scratch slot
  T* gscratch;            // per-CTA scratch for longer tubes: (NF + 5) * (nmax + 4) each
  int nmax;
  unsigned long long* cell_updates;  // running total
};

struct BatchPlan;
typedef void (*BatchLaunch)(const BatchPlan& pl, void* q, cudaStream_t st);

struct BatchPlan {
  HydroParams P{};
  double xmin = 0.0, xmax = 1.0;
  int nf = 5;
  long long ntot = 0;
  TubeState* tubes = nullptr;
  const int* order = nullptr;
  int ntubes = 0;
  int* head = nullptr;
  int budget = 1;
  long long quantum = 0;
  int cap = 0;
  int capw = 0;        // set with smem: the longest tube whose w fits the shared memory
  void* gscratch = nullptr;
  int nmax = 0;
  unsigned long long* cell_updates = nullptr;
  int threads = 256;   // NT
  int ctas = 1;        // persistent grid
  size_t smem = 0;
};

#define EVORA_DECLARE_BATCH_NS(ns)                                                          \
  namespace ns {                                                                            \
  /* configures launch for nf fields and `threads` per CTA; sets plan->smem from cap */     \
  BatchLaunch batch_pick(int nf, int threads, BatchPlan* plan);                             \
  int batch_max_ctas_per_sm(int nf, int threads, size_t smem);                              \
  }
EVORA_DECLARE_BATCH_NS(f64)
EVORA_DECLARE_BATCH_NS(f64s)
EVORA_DECLARE_BATCH_NS(f32)
#undef EVORA_DECLARE_BATCH_NS

// Reference layout q(6, n) (FP64) <-> packed SoA tube storage.
void tube_from_aos(const double* aos, void* q, bool f32, long long ntot, long long off, long long n, int nf,
                   cudaStream_t st);
void tube_to_aos(const void* q, double* aos, bool f32, long long ntot, long long off, long long n, int nf,
                 double g1, cudaStream_t st);
// Instantiation dispatch by precision.
BatchLaunch batch_pick_for(int precision, int strict, int nf, int threads, BatchPlan* pl);
int batch_ctas_per_sm(int precision, int strict, int nf, int threads, size_t smem);

}  // namespace evora
