// fused_tma.cuh -- the fused 3D update for grids tiled by whole TX x TY
// tiles, with the halo planes staged by the Tensor Memory Accelerator.
//
// Same algorithm and per-cell arithmetic as the tile program of
// fused_kernel.cuh (primitives, ghost map, slopes and predictor, the x, y and
// z Riemann solves and the conservative update of muscl.f90:171-290 and
// riemann.f90, in one HBM pass), with the per-thread work laid out so that
// no runtime index arithmetic remains in the plane loop:
//
//   * one elected thread loads each halo'd plane of the conserved state
//     (TX+2*XOFF) x (TY+4) x NF into a two-stage shared-memory ring with one
//     cp.async.bulk.tensor per plane, completion signalled on an mbarrier;
//     the load of plane p is issued 1.5 plane iterations before its use.  The
//     tensor map covers this GPU's own state buffer only; no multicast.
//   * each thread converts the same halo cells of every plane (one or two
//     for the shipped tiles; offsets fixed at kernel start), solves the x
//     interface on its cell's left, the y interface below it and the z
//     interface above it; the TX + TY closing interfaces of a plane and the 2 (TX + TY) ring cells
//     go to fixed threads packed into as few warps as possible.
//   * ghost cells (tiles at the domain edge) are read through the boundary
//     index map (boundary.f90:26-113) instead of the stage: the tensor load
//     fills them with zeros.
//
// Every wait on an mbarrier is bounded by a clock budget; a CTA whose wait
// runs out raises EVORA_ERR_TIMEOUT, waits (bounded) for its loads in flight
// and leaves the plane loop with the rest of the CTA at the next barrier.
//
// The host emulation (EVORA_HOST_EMU) performs the tensor load as a plain
// copy by the issuing thread, so the schedule can be checked against the
// oracle on the CPU.
#pragma once

#include "fused_kernel.cuh"

// Barrier that also ORs a predicate over the CTA.  In the host emulation
// the waits never run out, so the predicate is always false there.
#ifdef EVORA_HOST_EMU
#define EV_SYNC_OR(pred) (EV_SYNC(), (void)(pred), 0)
#else
#define EV_SYNC_OR(pred) __syncthreads_or(pred)
#endif

#if !defined(EVORA_HOST_EMU)
#include <cuda.h>
#endif

namespace evora {
namespace EVORA_FNS {

// Shared memory of one CTA.  XOFF: the stage box starts XOFF cells left of
// the tile so that its first x coordinate times the element size is a
// multiple of 16 bytes (the tensor copy's rule); the ring reads from x
// offset XOFF - 2.
template <typename T, int NF, int TX, int TY>
struct TmaSmem {
  static constexpr int RX = TX + 4, RY = TY + 4;
  static constexpr int XOFF = sizeof(T) == 4 ? 4 : 2;
  static constexpr int SX = TX + 2 * XOFF;
  static constexpr int PL = RY * RX;    // cells per field of a ring plane
  static constexpr int SPL = RY * SX;   // cells per field of a stage
  static constexpr unsigned kStageBytes = (unsigned)(NF * SPL * sizeof(T));
  static_assert((SX * sizeof(T)) % 16 == 0, "tensor box rows are whole 16-byte units");
  static_assert(kStageBytes % 128 == 0, "stages stay 128-byte aligned");
  alignas(128) T raw[2][NF][RY][SX];   // tensor-load stages (conserved state)
  T w[3][5][RY][RX];                   // primitive ring: planes c, c+1, c+2
  T xf[2][5][TY][TX + 2];              // x face states of the tile and the x ring
  T yf[2][5][TY + 2][TX];              // y face states of the tile and the y ring
  T fx[NF][TY][TX + 1];                // x fluxes, interface i-1/2 at column i
  T fy[NF][TY + 1][TX];                // y fluxes, interface j-1/2 at row j
  T cfl[3][sizeof(T) == 4 ? TX * TY : 32];
  T dq[NF][TX * TY];                   // owned cells' state of the plane being updated
  unsigned long long bar[2];           // one mbarrier per stage
#if defined(EVORA_HOST_EMU)
  std::atomic<unsigned> emu_loads[2];  // emulation: completed loads per stage
#endif
};

#if defined(EVORA_HOST_EMU)
using TmaMap = const void*;   // the emulation copies from FusedArgs::qin
#else
using TmaMap = CUtensorMap;
#endif

__device__ __forceinline__ unsigned smem_addr(const void* p) {
#if defined(EVORA_HOST_EMU)
  (void)p;
  return 0;
#else
  return (unsigned)__cvta_generic_to_shared(p);
#endif
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
#if !defined(EVORA_HOST_EMU)
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
#else
  (void)bar;
#endif
}

#if defined(EVORA_HOST_EMU)
// Emulated barrier phase: load number `use` of a stage has completed once
// its counter passed it (the copies are made by the issuing thread).
inline bool emu_wait(std::atomic<unsigned>& done, unsigned use) {
  while (done.load(std::memory_order_acquire) <= use) std::this_thread::yield();
  return true;
}
#endif

// Makes the initialised barriers visible to the other threads and to the
// tensor-copy (async) proxy.
__device__ __forceinline__ void mbar_fence_init() {
#if !defined(EVORA_HOST_EMU)
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
#endif
}

// One bounded wait for the completion of phase `parity` of a barrier:
// false if the clock budget (about a second) ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
#if !defined(EVORA_HOST_EMU)
  const unsigned a = smem_addr(bar);
  const long long t0 = clock64();
  for (;;) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > (1ll << 31)) return false;
  }
#else
  (void)bar;
  (void)parity;
  return true;
#endif
}

// Thread 0: announce the stage's bytes on its barrier and start the tensor
// load of box (x0, y0, z, 0) of the 4D map (x, y, z, field).
template <typename T, int NF, int TX, int TY>
__device__ __forceinline__ void tma_plane(const FusedArgs<T>& A, const TmaMap& map, TmaSmem<T, NF, TX, TY>& sm,
                                          int stage, int x0, int y0, int z) {
  using S = TmaSmem<T, NF, TX, TY>;
#if !defined(EVORA_HOST_EMU)
  (void)A;
  const unsigned bar = smem_addr(&sm.bar[stage]);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(S::kStageBytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_addr(&sm.raw[stage][0][0][0])),
      "l"(reinterpret_cast<unsigned long long>(&map)), "r"(x0), "r"(y0), "r"(z), "r"(0), "r"(bar)
      : "memory");
#else
  (void)map;
  const int nx = A.P.nx, ny = A.P.ny;
  for (int f = 0; f < NF; ++f)
    for (int y = 0; y < S::RY; ++y)
      for (int x = 0; x < S::SX; ++x) {
        const int gx = x0 + x, gy = y0 + y;
        sm.raw[stage][f][y][x] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
                                     ? A.qin[f * A.n + ((int64_t)z * ny + gy) * nx + gx]
                                     : (T)0;
      }
  sm.emu_loads[stage].fetch_add(1, std::memory_order_release);
#endif
}

// cp.async of one element (4 or 8 bytes), global -> shared.
template <typename T>
__device__ __forceinline__ void copy_async_el(T* dst, const T* src) {
#if !defined(EVORA_HOST_EMU)
  const unsigned s = smem_addr(dst);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
#else
  *dst = *src;
#endif
}

// The tile program.  Requires nx % TX == 0, ny % TY == 0 and a 3D grid.
template <typename T, int NF, int TX, int TY, int ZC>
__device__ __forceinline__ void tma_tile(const FusedArgs<T>& A, const TmaMap& map, TmaSmem<T, NF, TX, TY>& sm,
                                         int tid, int bx, int by, int bz) {
  using S = TmaSmem<T, NF, TX, TY>;
  constexpr int NT = TX * TY;
  constexpr int RX = S::RX, RY = S::RY, SX = S::SX, PL = S::PL, SPL = S::SPL, XOFF = S::XOFF;
  constexpr int NH = RX * RY;                // halo'd plane cells
  constexpr int HPT = (NH + NT - 1) / NT;    // halo cells per thread
  static_assert(2 * (TX + TY) <= NT && TX + TY <= NT, "ring cells and closing interfaces fit the CTA");
  const HydroParams& P = A.P;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int zc = A.zc > 0 ? A.zc : ZC;
  const int X0 = bx * TX, Y0 = by * TY, Z0 = bz * zc;
  const int ze = nz - Z0 < zc ? nz - Z0 : zc;
  const int oi = tid % TX, oj = tid / TX;
  const int64_t n = A.n;
  const int64_t nxy = (int64_t)nx * ny;
  const Gas<T> c = Gas<T>::make(P);
  const bool de = NF == 6 && P.dualenergy != 0;
  unsigned err = 0;
  const int64_t own = (int64_t)(Y0 + oj) * nx + (X0 + oi);   // owned column within a plane

  if (ctl_skip(A.ctl)) {
    for (int z = Z0; z < Z0 + ze; ++z) {
      const int64_t idx = (int64_t)z * nxy + own;
#pragma unroll
      for (int f = 0; f < NF; ++f) A.qout[f * n + idx] = A.qin[f * n + idx];
    }
    return;
  }

  const double dtd = A.ctl->dt;
  const T dt2 = (T)(-0.5 * dtd);
  const T dtdx = (T)(dtd * P.dxinv), dtdy = (T)(dtd * P.dyinv), dtdz = (T)(dtd * P.dzinv);

  // ---- fixed per-thread work: halo cells, ring cell, closing interface
  int h_w[HPT], h_r[HPT];  // offsets in a ring plane and in a stage
  int h_g[HPT];            // >= 0: ghost cell, in-plane index of the mapped cell
  bool h_flip[HPT], h_on[HPT];
#pragma unroll
  for (int h = 0; h < HPT; ++h) {
    const int k = tid + h * NT;
    h_on[h] = k < NH;
    const int lx = k % RX, ly = k / RX;
    h_w[h] = ly * RX + lx;
    h_r[h] = ly * SX + lx + (XOFF - 2);
    const int gx = X0 - 2 + lx, gy = Y0 - 2 + ly;
    bool flip = false;
    h_g[h] = -1;
    if (h_on[h] && (gx < 0 || gx >= nx || gy < 0 || gy >= ny)) {
      const int mx = ghost_map(gx, nx, P.boundtype, 0, flip);
      const int my = ghost_map(gy, ny, P.boundtype, 1, flip);
      h_g[h] = my * nx + mx;
    }
    h_flip[h] = flip;
  }
  // ring cell of this thread (faces only): x ring at x = -1 / TX of rows
  // 0..TY-1, then y ring at y = -1 / TY of columns 0..TX-1
  int r_w = -1, r_x = 0, r_y = 0;
  bool r_xring = false;
  if (tid < 2 * (TX + TY)) {
    if (tid < 2 * TY) {
      r_xring = true;
      r_y = tid >> 1;
      r_x = (tid & 1) ? TX : -1;
    } else {
      r_x = (tid - 2 * TY) >> 1;
      r_y = ((tid - 2 * TY) & 1) ? TY : -1;
    }
    r_w = (r_y + 2) * RX + (r_x + 2);
  }
  const int own_w = (oj + 2) * RX + (oi + 2);
  // closing interface of this thread: x interface TX of row e (e < TY), or
  // y interface TY of column e - TY; given to the last threads of the CTA
  const int ecl = tid - (NT - (TX + TY));

  // ---- staging: plane index L = p - (Z0 - 2) for planes Z0-2 .. Z0+ze+1
  const int nload = ze + 4;
  auto plane_z = [&](int L) {
    bool fl = false;
    return ghost_map(Z0 - 2 + L, nz, P.boundtype, 2, fl);
  };
  auto issue = [&](int L) {
    if (tid == 0 && L < nload) tma_plane<T, NF, TX, TY>(A, map, sm, L & 1, X0 - XOFF, Y0 - 2, plane_z(L));
  };
  int timed_out = 0;
  // A: convert staged plane L into the ring plane wd
  auto convert = [&](int L, T* wd) {
#if defined(EVORA_HOST_EMU)
    emu_wait(sm.emu_loads[L & 1], (unsigned)(L >> 1));
#endif
    if (!mbar_wait(&sm.bar[L & 1], (unsigned)((L >> 1) & 1))) {
      timed_out = 1;
      err |= EVORA_ERR_TIMEOUT;
    }
    const T* st = &sm.raw[L & 1][0][0][0];
    const T* plane = A.qin + (int64_t)plane_z(L) * nxy;
#pragma unroll
    for (int h = 0; h < HPT; ++h) {
      if (!h_on[h]) continue;
      T qv[6], wv[5];
      if (h_g[h] >= 0) {
#pragma unroll
        for (int f = 0; f < NF; ++f) qv[f] = ld(plane + f * n + h_g[h]);
      } else {
#pragma unroll
        for (int f = 0; f < NF; ++f) qv[f] = st[f * SPL + h_r[h]];
      }
      prim_k(qv, wv, c, P, de, err);
      if (h_flip[h]) {
        wv[1] = -wv[1];
        wv[2] = -wv[2];
        wv[3] = -wv[3];
      }
#pragma unroll
      for (int f = 0; f < 5; ++f) wd[f * PL + h_w[h]] = wv[f];
    }
  };
  // B: face states of the owned cell (and the ring cell when `in`), from
  // ring planes wp, wc, wn (planes c-1, c, c+1)
  auto faces = [&](const T* wp, const T* wc, const T* wn, bool in, T* wzm, T* wzp) {
    {
      const T* p0 = wp + own_w;
      const T* c0 = wc + own_w;
      const T* n0 = wn + own_w;
      T wv[5], face[3][2][5];
      cell_faces_g<T, 3>(
          [&](int f, int dx, int dy, int dz) -> T {
            if (dz < 0) return p0[f * PL];
            if (dz > 0) return n0[f * PL];
            return c0[f * PL + dy * RX + dx];
          },
          P, dt2, wv, face);
      if (in) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          sm.xf[0][f][oj][oi + 1] = face[0][0][f];
          sm.xf[1][f][oj][oi + 1] = face[0][1][f];
          sm.yf[0][f][oj + 1][oi] = face[1][0][f];
          sm.yf[1][f][oj + 1][oi] = face[1][1][f];
        }
      }
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        wzm[f] = face[2][0][f];
        wzp[f] = face[2][1][f];
      }
    }
    if (in && r_w >= 0) {
      const T* p0 = wp + r_w;
      const T* c0 = wc + r_w;
      const T* n0 = wn + r_w;
      T wv[5], face[3][2][5];
      cell_faces_g<T, 3>(
          [&](int f, int dx, int dy, int dz) -> T {
            if (dz < 0) return p0[f * PL];
            if (dz > 0) return n0[f * PL];
            return c0[f * PL + dy * RX + dx];
          },
          P, dt2, wv, face);
      if (r_xring) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          sm.xf[0][f][r_y][r_x + 1] = face[0][0][f];
          sm.xf[1][f][r_y][r_x + 1] = face[0][1][f];
        }
      } else {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          sm.yf[0][f][r_y + 1][r_x] = face[1][0][f];
          sm.yf[1][f][r_y + 1][r_x] = face[1][1][f];
        }
      }
    }
  };
  // C: the x interface left of the owned cell, the y interface below it,
  // and the closing interface given to this thread
  auto solves_xy = [&]() {
    T wl[5], wr[5], fv[NF];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      wl[f] = sm.xf[1][f][oj][oi];
      wr[f] = sm.xf[0][f][oj][oi + 1];
    }
    riemann_k<T, NF, 1>(wl, wr, fv, P.solver, c, err);
#pragma unroll
    for (int f = 0; f < NF; ++f) sm.fx[f][oj][oi] = fv[f];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      wl[f] = sm.yf[1][f][oj][oi];
      wr[f] = sm.yf[0][f][oj + 1][oi];
    }
    riemann_k<T, NF, 2>(wl, wr, fv, P.solver, c, err);
#pragma unroll
    for (int f = 0; f < NF; ++f) sm.fy[f][oj][oi] = fv[f];
    if (ecl >= 0) {
      if (ecl < TY) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          wl[f] = sm.xf[1][f][ecl][TX];
          wr[f] = sm.xf[0][f][ecl][TX + 1];
        }
        riemann_k<T, NF, 1>(wl, wr, fv, P.solver, c, err);
#pragma unroll
        for (int f = 0; f < NF; ++f) sm.fx[f][ecl][TX] = fv[f];
      } else {
        const int col = ecl - TY;
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          wl[f] = sm.yf[1][f][TY][col];
          wr[f] = sm.yf[0][f][TY + 1][col];
        }
        riemann_k<T, NF, 2>(wl, wr, fv, P.solver, c, err);
#pragma unroll
        for (int f = 0; f < NF; ++f) sm.fy[f][TY][col] = fv[f];
      }
    }
  };
  auto zflux = [&](const T* lo_plane_upper, const T* hi_plane_lower, T* fz) {
    riemann_k<T, NF, 3>(lo_plane_upper, hi_plane_lower, fz, P.solver, c, err);
  };

  // next-step CFL maxima over the written cells (as the tile program of
  // fused_kernel.cuh)
  constexpr bool kSlots = sizeof(T) == 4;
  unsigned cerr = 0;
  T cm0 = (T)0, cm1 = (T)0, cm2 = (T)0;
  if constexpr (kSlots)
    if (A.cfl_next) sm.cfl[0][tid] = sm.cfl[1][tid] = sm.cfl[2][tid] = (T)0;
  T qacc[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) qacc[f] = (T)0;
  auto write_plane = [&](int z, const T* fz_lo, const T* fz_hi) {
    const int64_t idx = (int64_t)z * nxy + own;
    T qo[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      qo[f] = qacc[f] + dtdz * (fz_lo[f] - fz_hi[f]);
      A.qout[f * n + idx] = qo[f];
    }
    if (A.cfl_next) {
      T s[3];
      cfl_speeds<T, NF>(qo, P, de, cerr, s);
      if constexpr (kSlots) {
        if (s[0] > sm.cfl[0][tid]) sm.cfl[0][tid] = s[0];
        if (s[1] > sm.cfl[1][tid]) sm.cfl[1][tid] = s[1];
        if (s[2] > sm.cfl[2][tid]) sm.cfl[2][tid] = s[2];
      } else {
        if (s[0] > cm0) cm0 = s[0];
        if (s[1] > cm1) cm1 = s[1];
        if (s[2] > cm2) cm2 = s[2];
      }
    }
  };
  auto prefetch_own = [&](int z) {
    const int64_t idx = (int64_t)z * nxy + own;
#pragma unroll
    for (int f = 0; f < NF; ++f) copy_async_el(&sm.dq[f][tid], A.qin + f * n + idx);
    copy_async_commit();
  };
  auto update_xy = [&]() {
    copy_async_wait();
    T qv[6], wdummy[5];
#pragma unroll
    for (int f = 0; f < NF; ++f) qv[f] = sm.dq[f][tid];
    if (de) {
      unsigned e2 = 0;
      prim_k(qv, wdummy, c, P, de, e2);   // dual-energy resync of q (comp.f90:60-72)
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) qv[f] = qv[f] + dtdx * (sm.fx[f][oj][oi] - sm.fx[f][oj][oi + 1]);
#pragma unroll
    for (int f = 0; f < NF; ++f) qacc[f] = qv[f] + dtdy * (sm.fy[f][oj][oi] - sm.fy[f][oj + 1][oi]);
  };

  T* const ring0 = &sm.w[0][0][0][0];
  constexpr int kRing = 5 * PL;
  // ---- prologue: planes Z0-2 .. Z0+1 into ring slots L % 3
  if (tid == 0) {
    mbar_init(&sm.bar[0]);
    mbar_init(&sm.bar[1]);
    mbar_fence_init();
#if defined(EVORA_HOST_EMU)
    sm.emu_loads[0] = 0;
    sm.emu_loads[1] = 0;
#endif
  }
  EV_SYNC();
  issue(0);
  issue(1);
  convert(0, ring0);
  EV_SYNC();
  issue(2);
  convert(1, ring0 + kRing);
  EV_SYNC();
  issue(3);
  convert(2, ring0 + 2 * kRing);
  EV_SYNC();
  issue(4);
  T wzm_n[5], wzp_n[5], wzp_c[5], fz_cur[NF], fz_prev[NF];
  faces(ring0, ring0 + kRing, ring0 + 2 * kRing, false, wzm_n, wzp_c);   // plane Z0-1: z faces only
  EV_SYNC();
  convert(3, ring0);                                                        // plane Z0+1
  EV_SYNC();
  issue(5);
  faces(ring0 + kRing, ring0 + 2 * kRing, ring0, true, wzm_n, wzp_n);     // plane Z0
  zflux(wzp_c, wzm_n, fz_cur);                                             // Z0 - 1/2
#pragma unroll
  for (int f = 0; f < 5; ++f) wzp_c[f] = wzp_n[f];
#pragma unroll
  for (int f = 0; f < NF; ++f) fz_prev[f] = (T)0;
  // a wait that ran out (any thread) ends the march for the whole CTA
  bool ok = !EV_SYNC_OR(timed_out);
  int issued = 5;   // planes whose loads were started (L < issued)
  // ring planes of cz, cz+1, cz+2
  T* sa = ring0 + 2 * kRing;
  T* sb = ring0;
  T* sc = ring0 + kRing;
  int converted = 4;   // planes converted (L < converted)
  for (int cz = Z0; ok && cz < Z0 + ze; ++cz) {
    const int L = cz - Z0 + 4;
    // ---- I1: A(cz+2), x/y solves of plane cz
    prefetch_own(cz);
    convert(L, sc);
    converted = L + 1;
    solves_xy();
    EV_SYNC();
    issue(L + 2);
    issued = L + 3;
    // ---- I2: plane cz-1 out, plane cz's x/y terms, B(cz+1), flux cz+1/2
    if (cz > Z0) write_plane(cz - 1, fz_prev, fz_cur);
    update_xy();
    faces(sa, sb, sc, cz + 1 < Z0 + ze, wzm_n, wzp_n);
#pragma unroll
    for (int f = 0; f < NF; ++f) fz_prev[f] = fz_cur[f];
    zflux(wzp_c, wzm_n, fz_cur);
#pragma unroll
    for (int f = 0; f < 5; ++f) wzp_c[f] = wzp_n[f];
    T* t = sa;
    sa = sb;
    sb = sc;
    sc = t;
    ok = !EV_SYNC_OR(timed_out);
  }
  if (ok) {
    write_plane(Z0 + ze - 1, fz_prev, fz_cur);
  } else if (tid == 0) {
    // a wait ran out: wait (bounded) for the loads still in flight, so that
    // no tensor copy lands in this CTA's shared memory after it exits
    for (int L = converted; L < issued && L < nload; ++L) mbar_wait(&sm.bar[L & 1], (unsigned)((L >> 1) & 1));
  }
  if (err) {
#if defined(EVORA_HOST_EMU)
    reinterpret_cast<std::atomic<unsigned>*>(&A.ctl->err)->fetch_or(err);
#else
    atomicOr(&A.ctl->err, err);
#endif
  }
  if (!ok) return;   // uniform: every thread read the same abort flag
  if (A.cfl_next) {
    if constexpr (kSlots) {
      cm0 = sm.cfl[0][tid];
      cm1 = sm.cfl[1][tid];
      cm2 = sm.cfl[2][tid];
    }
#if defined(EVORA_HOST_EMU)
    const double cm[3] = {cm0, cm1, cm2};
    for (int d = 0; d < 3; ++d) {
      std::atomic_ref<unsigned long long> r(A.ctl->snext[d]);
      unsigned long long cur = r.load(), v = ordered_bits(cm[d]);
      while (v > cur && !r.compare_exchange_weak(cur, v)) {
      }
    }
    if (cerr) std::atomic_ref<unsigned>(A.ctl->errnext).fetch_or(cerr);
#else
    for (int o = 16; o > 0; o >>= 1) {
      cm0 = fmax2(cm0, __shfl_xor_sync(0xffffffffu, cm0, o));
      cm1 = fmax2(cm1, __shfl_xor_sync(0xffffffffu, cm1, o));
      cm2 = fmax2(cm2, __shfl_xor_sync(0xffffffffu, cm2, o));
    }
    EV_SYNC();
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) {
      sm.cfl[0][wid] = cm0;
      sm.cfl[1][wid] = cm1;
      sm.cfl[2][wid] = cm2;
    }
    EV_SYNC();
    if (tid == 0) {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int k = 0; k < NT / 32; ++k) {
        a0 = fmax2(a0, (double)sm.cfl[0][k]);
        a1 = fmax2(a1, (double)sm.cfl[1][k]);
        a2 = fmax2(a2, (double)sm.cfl[2][k]);
      }
      atomicMax(&A.ctl->snext[0], ordered_bits(a0));
      atomicMax(&A.ctl->snext[1], ordered_bits(a1));
      atomicMax(&A.ctl->snext[2], ordered_bits(a2));
    }
    if (cerr) atomicOr(&A.ctl->errnext, cerr);
#endif
  }
}

#if !defined(EVORA_HOST_EMU)
template <typename T, int NF, int TX, int TY, int ZC, int MINB>
__global__ void __launch_bounds__(TX* TY, MINB) k_fused_tma(FusedArgs<T> A, const __grid_constant__ CUtensorMap map) {
  extern __shared__ __align__(128) unsigned char smem_staged[];
  auto& sm = *reinterpret_cast<TmaSmem<T, NF, TX, TY>*>(smem_staged);
  tma_tile<T, NF, TX, TY, ZC>(A, map, sm, threadIdx.x, blockIdx.x, blockIdx.y, blockIdx.z);
}
#endif

}  // namespace EVORA_FNS
}  // namespace evora
