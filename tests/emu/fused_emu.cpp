// Host emulation of the fused CUDA kernels (test harness): the tile program
// of evora_b200/csrc/fused_kernel.cuh compiled with g++, each CTA's threads
// run as std::threads meeting at a std::barrier.  With -ffp-contract=off
// the arithmetic is the reference's, so its output must equal the CPU oracle
// bit for bit; a difference points at the tiling, halo or boundary logic.
#define EVORA_HOST_EMU 1
#include <atomic>
#include <thread>
#define EVORA_FNS emu
#include "../../evora_b200/csrc/fused_kernel.cuh"
#include "../../evora_b200/csrc/fused_tma.cuh"
#include "../../evora_b200/csrc/fused_pair.cuh"

#include <cstring>
#include <memory>
#include <thread>
#include <vector>

thread_local std::barrier<>* evora_emu::tl_barrier = nullptr;

using namespace evora;
using namespace evora::emu;

// 1: the two-barrier pipelined 3D march (the FP32 kernels' schedule),
// 0: the three-barrier march (the FP64 kernels' schedule),
// 2: the tensor-staged march of fused_tma.cuh (3D grids of whole tiles; the
//    tensor load is a copy by the issuing thread),
// 3: the two-cells-per-thread march of fused_pair.cuh (fast-form arithmetic
//    in FP64 here: equal to the oracle up to rounding, not bit for bit)
static int g_pipe = 0;
extern "C" void emu_set_pipeline(int on) { g_pipe = on; }
// planes per CTA of the 3D march (0: the tile's ZC)
static int g_zc = 0;
extern "C" void emu_set_zc(int zc) { g_zc = zc; }

template <int NF, int TX, int TY, int ZC>
static void run_tma_tiles(const FusedArgs<double>& A) {
  constexpr int NT = TX * TY;
  const HydroParams& P = A.P;
  const int zc = A.zc > 0 ? A.zc : ZC;
  const int gx = P.nx / TX, gy = P.ny / TY, gz = (P.nz + zc - 1) / zc;
  auto sm = std::make_unique<TmaSmem<double, NF, TX, TY>>();
  const void* map = nullptr;
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        std::barrier<> bar(NT);
        std::vector<std::thread> th;
        th.reserve(NT);
        for (int t = 0; t < NT; ++t)
          th.emplace_back([&, t] {
            evora_emu::tl_barrier = &bar;
            tma_tile<double, NF, TX, TY, ZC>(A, map, *sm, t, bx, by, bz);
          });
        for (auto& x : th) x.join();
      }
}

template <int TX, int TY, int ZC>
static void run_pair_tiles(const FusedArgs<double>& A) {
  constexpr int NT = TX / 2 * TY;
  const HydroParams& P = A.P;
  const int zc = A.zc > 0 ? A.zc : ZC;
  const int gx = P.nx / TX, gy = P.ny / TY, gz = (P.nz + zc - 1) / zc;
  auto sm = std::make_unique<PairSmem<double, TX, TY>>();
  const void* map = nullptr;
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        std::barrier<> bar(NT);
        std::vector<std::thread> th;
        th.reserve(NT);
        for (int t = 0; t < NT; ++t)
          th.emplace_back([&, t] {
            evora_emu::tl_barrier = &bar;
            pair_tile<double, TX, TY, ZC>(A, map, *sm, t, bx, by, bz);
          });
        for (auto& x : th) x.join();
      }
}

template <int NF, int DIM, int TX, int TY, int ZC>
static void run_tiles(const FusedArgs<double>& A) {
  if constexpr (DIM == 3) {
    if (g_pipe == 2 && A.P.nx % TX == 0 && A.P.ny % TY == 0) {
      run_tma_tiles<NF, TX, TY, ZC>(A);
      return;
    }
    if constexpr (NF == 5 && TX % 16 == 0 && TX / 2 * TY >= 2 * (TX / 2 + TY)) {
      if (g_pipe == 3 && A.P.nx % TX == 0 && A.P.ny % TY == 0 && pair_config(A.P)) {
        run_pair_tiles<TX, TY, ZC>(A);
        return;
      }
    }
  }
  constexpr int NT = TX * TY;
  const HydroParams& P = A.P;
  const int gx = (P.nx + TX - 1) / TX, gy = (P.ny + TY - 1) / TY;
  const int gz = DIM == 3 ? (P.nz + ZC - 1) / ZC : 1;
  auto sm = std::make_unique<FusedSmem<double, NF, TX, TY>>();
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx) {
        std::barrier<> bar(NT);
        std::vector<std::thread> th;
        th.reserve(NT);
        for (int t = 0; t < NT; ++t)
          th.emplace_back([&, t] {
            evora_emu::tl_barrier = &bar;
            if (g_pipe) fused_tile<double, NF, DIM, TX, TY, ZC, true>(A, *sm, t, bx, by, bz);
            else fused_tile<double, NF, DIM, TX, TY, ZC, false>(A, *sm, t, bx, by, bz);
          });
        for (auto& x : th) x.join();
      }
}

// smax_next (may be null): the next step's CFL maxima that the update
// reduces over the state it writes (2D and 3D tiles), as doubles.
extern "C" int emu_fused_update_cfl(const HydroParams* P, int nf, const double* qin, double* qout, double dt,
                                    int tile, double* smax_next) {
  GridCtl ctl{};
  ctl.dt = dt;
  ctl.go = 1;
  ctl.active = 1;
  const int dim = P->onedimension ? 1 : (P->twodimension ? 2 : 3);
  FusedArgs<double> A{*P, qin, qout, &ctl, (int64_t)P->nx * P->ny * P->nz, smax_next != nullptr ? 1 : 0, g_zc};
  struct Out {
    GridCtl& c;
    double* s;
    ~Out() {
      if (s)
        for (int d = 0; d < 3; ++d) std::memcpy(&s[d], &c.snext[d], sizeof(double));
    }
  } out{ctl, smax_next};
  if (dim == 1) {
    for (int i = 0; i < P->nx; ++i) {
      if (nf == 5) fused_cell1d<double, 5>(A, i);
      else fused_cell1d<double, 6>(A, i);
    }
    return (int)ctl.err;
  }
#define RUN(NF, DIM)                                            \
  do {                                                          \
    if (tile == 0) run_tiles<NF, DIM, 8, 4, 4>(A);              \
    else if (tile == 1) run_tiles<NF, DIM, 32, 4, 32>(A);       \
    else run_tiles<NF, DIM, 16, 8, 4>(A);                       \
  } while (0)
  if (nf == 5 && dim == 2) RUN(5, 2);
  else if (nf == 5) RUN(5, 3);
  else if (dim == 2) RUN(6, 2);
  else RUN(6, 3);
#undef RUN
  return (int)ctl.err;
}

extern "C" int emu_fused_update(const HydroParams* P, int nf, const double* qin, double* qout, double dt,
                                int tile) {
  return emu_fused_update_cfl(P, nf, qin, qout, dt, tile, nullptr);
}
