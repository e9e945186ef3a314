// fused_pair.cuh -- the FP32 fused 3D update with two cells per thread.
//
// The algorithm is that of fused_kernel.cuh and fused_tma.cuh: one HBM pass
// per step that recovers the primitives of a halo'd plane, takes slopes and
// the predictor, solves every x, y and z interface once and applies the
// conservative update (muscl.f90:171-290, riemann.f90:96-205), marching a
// TX x TY column tile up a chunk of z planes.  Here a thread owns the two
// cells x and x + TX/2 of a row of the tile, so that the per-cell arithmetic
// of pair_math.cuh runs on packed FP32 pairs (one f32x2 instruction for two
// cells) and shared-memory traffic moves 8-byte pairs:
//
//   * the halo'd plane is staged by one tensor load per plane into a
//     two-stage mbarrier ring (as fused_tma.cuh; this GPU's own state only,
//     no multicast) and converted into a primitive ring held as pairs;
//   * x face states and x fluxes pass between neighbouring pairs of a row by
//     warp shuffles (a row of TX/2 pairs is a shuffle segment), y faces and
//     y fluxes through shared memory, z faces and fluxes stay in registers;
//   * the x ring (pairs -1 and TX/2), the y ring and the closing interfaces
//     go to fixed threads packed into as few warps as possible.
//
// Taken for FP32 grids of whole tiles with 5 fields, HLLC, minmod and the
// second-order scheme (the benchmark's configuration); other grids use the
// other tile entries.  The host emulation (EVORA_HOST_EMU, S = double) runs
// the same schedule with plain arithmetic; shuffles become exchanges through
// a buffer between two barriers.
#pragma once

#include "fused_tma.cuh"
#include "pair_math.cuh"

namespace evora {
namespace EVORA_FNS {

template <typename S, int TX, int TY>
struct PairSmem {
  static constexpr int HX = TX / 2;          // pairs per row
  static constexpr int NT = HX * TY;         // threads
  static constexpr int RX2 = HX + 4;         // pair columns of a ring plane: pairs -2 .. HX+1
  static constexpr int RY = TY + 4;
  static constexpr int XOFF = sizeof(S) == 4 ? 4 : 2;
  static constexpr int SX = TX + 2 * XOFF;   // stage row (cells), as fused_tma.cuh
  static constexpr int SPL = RY * SX;
  static constexpr int PL2 = RY * RX2;
  static constexpr unsigned kStageBytes = (unsigned)(5 * SPL * sizeof(S));
  static_assert((SX * sizeof(S)) % 16 == 0 && kStageBytes % 128 == 0, "tensor box alignment");
  alignas(128) S raw[2][5][RY][SX];   // tensor-load stages (conserved state, cells)
  P2<S> w[3][5][RY][RX2];             // primitive ring: planes c, c+1, c+2 (pairs)
  P2<S> yu[5][TY + 1][HX];            // upper y faces of rows -1 .. TY-1 (row r at r + 1)
  P2<S> ylr[5][HX];                   // lower y faces of the ring row TY
  P2<S> xrl[5][TY];                   // upper x faces of pair -1 (cells -1, HX-1)
  P2<S> xrh[5][TY];                   // lower x faces of pair HX (cells HX, TX)
  P2<S> xul[5][TY];                   // upper x faces of pair HX-1 (cells HX-1, TX-1)
  P2<S> fy[5][TY + 1][HX];            // y fluxes, interface r-1/2 at row r
  S fxc[5][TY];                       // x flux through interface TX-1/2 of each row
  P2<S> dq[5][NT];                    // owned cells' state of the plane being updated
  S cfl[3][NT / 32 > 0 ? NT / 32 : 1];
  unsigned long long bar[2];
#if defined(EVORA_HOST_EMU)
  std::atomic<unsigned> emu_loads[2];
  P2<S> emu_x[5][NT];                 // emulated shuffles
#endif
};

// Thread 0: the tensor load of one staged plane (fields 0..4).
template <typename S, int TX, int TY>
__device__ __forceinline__ void pair_tma_plane(const FusedArgs<S>& A, const TmaMap& map, PairSmem<S, TX, TY>& sm,
                                               int stage, int x0, int y0, int z) {
  using PS = PairSmem<S, TX, TY>;
#if !defined(EVORA_HOST_EMU)
  (void)A;
  const unsigned bar = smem_addr(&sm.bar[stage]);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(PS::kStageBytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_addr(&sm.raw[stage][0][0][0])),
      "l"(reinterpret_cast<unsigned long long>(&map)), "r"(x0), "r"(y0), "r"(z), "r"(0), "r"(bar)
      : "memory");
#else
  (void)map;
  const int nx = A.P.nx, ny = A.P.ny;
  for (int f = 0; f < 5; ++f)
    for (int y = 0; y < PS::RY; ++y)
      for (int x = 0; x < PS::SX; ++x) {
        const int gx = x0 + x, gy = y0 + y;
        sm.raw[stage][f][y][x] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
                                     ? A.qin[f * A.n + ((int64_t)z * ny + gy) * nx + gx]
                                     : (S)0;
      }
  sm.emu_loads[stage].fetch_add(1, std::memory_order_release);
#endif
}

// Whether the pair kernel takes a grid (besides whole tiles).
__host__ __device__ inline bool pair_config(const HydroParams& P) {
  return P.solver == 2 && P.limiter == 1 && P.secondorder && !P.dualenergy;
}

template <typename S, int TX, int TY, int ZC>
__device__ __forceinline__ void pair_tile(const FusedArgs<S>& A, const TmaMap& map, PairSmem<S, TX, TY>& sm,
                                          int tid, int bx, int by, int bz) {
  using PS = PairSmem<S, TX, TY>;
  using V = P2<S>;
  constexpr int HX = PS::HX, NT = PS::NT, RX2 = PS::RX2, RY = PS::RY, SX = PS::SX, SPL = PS::SPL, PL2 = PS::PL2;
  constexpr int XOFF = PS::XOFF;
  constexpr int NH = RX2 * RY;                 // pair cells of a halo'd plane
  constexpr int HPT = (NH + NT - 1) / NT;
  static_assert(HX == 8 || HX == 16 || HX == 32, "a row of pairs is a shuffle segment");
  static_assert(2 * (TY + HX) <= NT && TY + HX <= NT, "ring cells and closing interfaces fit the CTA");
  const HydroParams& P = A.P;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int zc = A.zc > 0 ? A.zc : ZC;
  const int X0 = bx * TX, Y0 = by * TY, Z0 = bz * zc;
  const int ze = nz - Z0 < zc ? nz - Z0 : zc;
  const int p = tid % HX, j = tid / HX;      // owned pair: cells (p, j) and (p + HX, j) of the tile
  const int64_t n = A.n;
  const int64_t nxy = (int64_t)nx * ny;
  const Gas<S> c = Gas<S>::make(P);
  unsigned err = 0;
  const int64_t own = (int64_t)(Y0 + j) * nx + (X0 + p);
  // tiles whose x/y halo lies inside the grid read every halo cell from the
  // staged plane: no ghost map, no reflection (a block-uniform branch)
  const bool edge = !(X0 >= 2 && X0 + TX + 2 <= nx && Y0 >= 2 && Y0 + TY + 2 <= ny);

  if (ctl_skip(A.ctl)) {
    for (int z = Z0; z < Z0 + ze; ++z) {
      const int64_t idx = (int64_t)z * nxy + own;
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        A.qout[f * n + idx] = A.qin[f * n + idx];
        A.qout[f * n + idx + HX] = A.qin[f * n + idx + HX];
      }
    }
    return;
  }

  const double dtd = A.ctl->dt;
  const S dt2 = (S)(-0.5 * dtd);
  const V dtdx = p2<S>((S)(dtd * P.dxinv)), dtdy = p2<S>((S)(dtd * P.dyinv)), dtdz = p2<S>((S)(dtd * P.dzinv));

  // ---- fixed per-thread work
  // halo pair cells: item k = (row r, pair column pc), both cells
  int h_r[HPT][2], h_g[HPT][2];
  bool h_on[HPT], h_flip[HPT][2];
#pragma unroll
  for (int h = 0; h < HPT; ++h) {
    const int k = tid + h * NT;
    h_on[h] = k < NH;
    const int pc = k % RX2 - 2, r = k / RX2 - 2;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = pc + e * HX;
      h_r[h][e] = (r + 2) * SX + x + XOFF;
      const int gx = X0 + x, gy = Y0 + r;
      bool flip = false;
      h_g[h][e] = -1;
      if (h_on[h] && (gx < 0 || gx >= nx || gy < 0 || gy >= ny)) {
        const int mx = ghost_map(gx, nx, P.boundtype, 0, flip);
        const int my = ghost_map(gy, ny, P.boundtype, 1, flip);
        h_g[h][e] = my * nx + mx;
      }
      h_flip[h][e] = flip;
    }
  }
  // ring pair of this thread: x ring (pairs -1 and HX of rows 0..TY-1), then
  // y ring (rows -1 and TY of pairs 0..HX-1)
  int r_w = -1, r_a = 0, r_b = 0, r_kind = 0;   // kind 0 pair -1, 1 pair HX, 2 row -1, 3 row TY
  if (tid < 2 * (TY + HX)) {
    if (tid < 2 * TY) {
      r_b = tid >> 1;                      // row
      r_kind = tid & 1;
      r_a = r_kind ? HX : -1;              // pair column
    } else {
      r_a = (tid - 2 * TY) >> 1;
      r_kind = 2 + ((tid - 2 * TY) & 1);
      r_b = r_kind == 3 ? TY : -1;
    }
    r_w = (r_b + 2) * RX2 + (r_a + 2);
  }
  const int own_w = (j + 2) * RX2 + (p + 2);
  const int ecl = tid - (NT - (TY + HX));   // closing interface: x of row ecl, or y of pair ecl - TY

  // ---- staging (plane index L = p - (Z0 - 2))
  const int nload = ze + 4;
  auto plane_z = [&](int L) {
    bool fl = false;
    return ghost_map(Z0 - 2 + L, nz, P.boundtype, 2, fl);
  };
  auto issue = [&](int L) {
    if (tid == 0 && L < nload) pair_tma_plane<S, TX, TY>(A, map, sm, L & 1, X0 - XOFF, Y0 - 2, plane_z(L));
  };
  int timed_out = 0;
  auto convert = [&](int L, V* wd) {
#if defined(EVORA_HOST_EMU)
    emu_wait(sm.emu_loads[L & 1], (unsigned)(L >> 1));
#endif
    if (!mbar_wait(&sm.bar[L & 1], (unsigned)((L >> 1) & 1))) {
      timed_out = 1;
      err |= EVORA_ERR_TIMEOUT;
    }
    const S* st = &sm.raw[L & 1][0][0][0];
    const S* plane = A.qin + (int64_t)plane_z(L) * nxy;
#pragma unroll
    for (int h = 0; h < HPT; ++h) {
      if (!h_on[h]) continue;
      V qv[5], wv[5];
      if (edge) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          qv[f].x = h_g[h][0] >= 0 ? ld(plane + f * n + h_g[h][0]) : st[f * SPL + h_r[h][0]];
          qv[f].y = h_g[h][1] >= 0 ? ld(plane + f * n + h_g[h][1]) : st[f * SPL + h_r[h][1]];
        }
      } else {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          qv[f].x = st[f * SPL + h_r[h][0]];
          qv[f].y = st[f * SPL + h_r[h][1]];
        }
      }
      prim_p(qv, wv, c, P, err);
      if (edge && h_flip[h][0]) {
        wv[1].x = -wv[1].x;
        wv[2].x = -wv[2].x;
        wv[3].x = -wv[3].x;
      }
      if (edge && h_flip[h][1]) {
        wv[1].y = -wv[1].y;
        wv[2].y = -wv[2].y;
        wv[3].y = -wv[3].y;
      }
      const int k = tid + h * NT;
#pragma unroll
      for (int f = 0; f < 5; ++f) wd[f * PL2 + k] = wv[f];
    }
  };

  // ---- faces (B): owned pair into registers (x lower / upper, y lower) and
  // shared memory (y upper; the upper x face of pair HX-1), ring pair into
  // shared memory; z faces returned
  V xl[5], xu[5], yl[5];
  auto faces = [&](const V* wp, const V* wc, const V* wn, bool in, V* wzm, V* wzp) {
    {
      const V* p0 = wp + own_w;
      const V* c0 = wc + own_w;
      const V* n0 = wn + own_w;
      V wv[5], face[3][2][5];
      faces_p<S>(
          [&](int f, int dx, int dy, int dz) -> V {
            if (dz < 0) return p0[f * PL2];
            if (dz > 0) return n0[f * PL2];
            return c0[f * PL2 + dy * RX2 + dx];
          },
          P, dt2, wv, face);
      if (in) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          xl[f] = face[0][0][f];
          xu[f] = face[0][1][f];
          yl[f] = face[1][0][f];
          sm.yu[f][j + 1][p] = face[1][1][f];
        }
        if (p == HX - 1) {
#pragma unroll
          for (int f = 0; f < 5; ++f) sm.xul[f][j] = face[0][1][f];
        }
      }
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        wzm[f] = face[2][0][f];
        wzp[f] = face[2][1][f];
      }
    }
    if (in && r_w >= 0) {
      const V* p0 = wp + r_w;
      const V* c0 = wc + r_w;
      const V* n0 = wn + r_w;
      V wv[5], face[3][2][5];
      faces_p<S>(
          [&](int f, int dx, int dy, int dz) -> V {
            if (dz < 0) return p0[f * PL2];
            if (dz > 0) return n0[f * PL2];
            return c0[f * PL2 + dy * RX2 + dx];
          },
          P, dt2, wv, face);
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        if (r_kind == 0) sm.xrl[f][r_b] = face[0][1][f];
        else if (r_kind == 1) sm.xrh[f][r_b] = face[0][0][f];
        else if (r_kind == 2) sm.yu[f][0][r_a] = face[1][1][f];
        else sm.ylr[f][r_a] = face[1][0][f];
      }
    }
  };

  // ---- exchanges between the pairs of a row (a shuffle segment)
  auto from_left = [&](V* v) {   // v of pair p-1 (pair 0 keeps its own)
#if defined(EVORA_HOST_EMU)
    for (int f = 0; f < 5; ++f) sm.emu_x[f][tid] = v[f];
    EV_SYNC();
    V r[5];
    for (int f = 0; f < 5; ++f) r[f] = p > 0 ? sm.emu_x[f][tid - 1] : v[f];
    EV_SYNC();
    for (int f = 0; f < 5; ++f) v[f] = r[f];
#else
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      v[f].x = __shfl_up_sync(0xffffffffu, v[f].x, 1, HX);
      v[f].y = __shfl_up_sync(0xffffffffu, v[f].y, 1, HX);
    }
#endif
  };
  auto from_right = [&](const V* v, V* r) {   // v of pair (p + 1) mod HX
#if defined(EVORA_HOST_EMU)
    for (int f = 0; f < 5; ++f) sm.emu_x[f][tid] = v[f];
    EV_SYNC();
    const int src = j * HX + (p + 1) % HX;
    for (int f = 0; f < 5; ++f) r[f] = sm.emu_x[f][src];
    EV_SYNC();
#else
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      r[f].x = __shfl_sync(0xffffffffu, v[f].x, (p + 1) % HX, HX);
      r[f].y = __shfl_sync(0xffffffffu, v[f].y, (p + 1) % HX, HX);
    }
#endif
  };

  // ---- C: x and y solves of a plane (faces from the previous interval)
  V fxl[5], fxr[5];
  auto solves_xy = [&]() {
    // left states of both solves first, then the two solves as one
    // straight-line block (independent chains the scheduler interleaves)
    V wl[5], wly[5], fv[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) wl[f] = xu[f];
    from_left(wl);
    const M2 first{p == 0, p == 0};
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      wl[f] = sel2(first, sm.xrl[f][j], wl[f]);
      wly[f] = sm.yu[f][j][p];
    }
    hllc_p<S, 1>(wl, xl, fxl, c, err);
    hllc_p<S, 2>(wly, yl, fv, c, err);
#pragma unroll
    for (int f = 0; f < 5; ++f) sm.fy[f][j][p] = fv[f];
    // the flux right of the pair: .x through (p, p+1), .y through (p+HX,
    // p+HX+1); pair HX-1 takes .x from pair 0's .y and .y from the closing
    // interface (in the update)
    V fr[5];
    from_right(fxl, fr);
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      fxr[f].x = p < HX - 1 ? fr[f].x : fr[f].y;
      fxr[f].y = fr[f].y;
    }
    if (ecl >= 0) {
      V wr[5];
      if (ecl < TY) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          wl[f] = sm.xul[f][ecl];
          wr[f] = sm.xrh[f][ecl];
        }
        hllc_p<S, 1>(wl, wr, fv, c, err);
#pragma unroll
        for (int f = 0; f < 5; ++f) sm.fxc[f][ecl] = fv[f].y;
      } else {
        const int pc = ecl - TY;
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          wl[f] = sm.yu[f][TY][pc];
          wr[f] = sm.ylr[f][pc];
        }
        hllc_p<S, 2>(wl, wr, fv, c, err);
#pragma unroll
        for (int f = 0; f < 5; ++f) sm.fy[f][TY][pc] = fv[f];
      }
    }
  };

  // next-step CFL maxima over the written cells
  unsigned cerr = 0;
  S cm0 = (S)0, cm1 = (S)0, cm2 = (S)0;
  V qacc[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) qacc[f] = p2<S>((S)0);
  auto write_plane = [&](int z, const V* fz_lo, const V* fz_hi) {
    const int64_t idx = (int64_t)z * nxy + own;
    V qo[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      qo[f] = fma2(dtdz, fz_lo[f] - fz_hi[f], qacc[f]);
      A.qout[f * n + idx] = qo[f].x;
      A.qout[f * n + idx + HX] = qo[f].y;
    }
    if (A.cfl_next) {
      V s[3];
      speeds_p(qo, c, P, cerr, s);
      cm0 = fmax2(cm0, fmax2(s[0].x, s[0].y));
      cm1 = fmax2(cm1, fmax2(s[1].x, s[1].y));
      cm2 = fmax2(cm2, fmax2(s[2].x, s[2].y));
    }
  };
  auto prefetch_own = [&](int z) {
    const int64_t idx = (int64_t)z * nxy + own;
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      copy_async_el(&sm.dq[f][tid].x, A.qin + f * n + idx);
      copy_async_el(&sm.dq[f][tid].y, A.qin + f * n + idx + HX);
    }
    copy_async_commit();
  };
  auto update_xy = [&]() {
    copy_async_wait();
    if (p == HX - 1) {
#pragma unroll
      for (int f = 0; f < 5; ++f) fxr[f].y = sm.fxc[f][j];
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const V qx = fma2(dtdx, fxl[f] - fxr[f], sm.dq[f][tid]);
      qacc[f] = fma2(dtdy, sm.fy[f][j][p] - sm.fy[f][j + 1][p], qx);
    }
  };
  auto zflux = [&](const V* lo_plane_upper, const V* hi_plane_lower, V* fz) {
    hllc_p<S, 3>(lo_plane_upper, hi_plane_lower, fz, c, err);
  };

  V* const ring0 = &sm.w[0][0][0][0];
  constexpr int kRing = 5 * PL2;
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
  V wzm_n[5], wzp_n[5], wzp_c[5], fz_cur[5], fz_prev[5];
  faces(ring0, ring0 + kRing, ring0 + 2 * kRing, false, wzm_n, wzp_c);   // plane Z0-1: z faces only
  EV_SYNC();
  convert(3, ring0);                                                        // plane Z0+1
  EV_SYNC();
  issue(5);
  faces(ring0 + kRing, ring0 + 2 * kRing, ring0, true, wzm_n, wzp_n);     // plane Z0
  zflux(wzp_c, wzm_n, fz_cur);                                             // Z0 - 1/2
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    wzp_c[f] = wzp_n[f];
    fz_prev[f] = p2<S>((S)0);
  }
  bool ok = !EV_SYNC_OR(timed_out);
  int issued = 5, converted = 4;
  V* sa = ring0 + 2 * kRing;
  V* sb = ring0;
  V* sc = ring0 + kRing;
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
    for (int f = 0; f < 5; ++f) fz_prev[f] = fz_cur[f];
    zflux(wzp_c, wzm_n, fz_cur);
#pragma unroll
    for (int f = 0; f < 5; ++f) wzp_c[f] = wzp_n[f];
    V* t = sa;
    sa = sb;
    sb = sc;
    sc = t;
    ok = !EV_SYNC_OR(timed_out);
  }
  if (ok) {
    write_plane(Z0 + ze - 1, fz_prev, fz_cur);
  } else if (tid == 0) {
    for (int L = converted; L < issued && L < nload; ++L) mbar_wait(&sm.bar[L & 1], (unsigned)((L >> 1) & 1));
  }
  if (err) {
#if defined(EVORA_HOST_EMU)
    reinterpret_cast<std::atomic<unsigned>*>(&A.ctl->err)->fetch_or(err);
#else
    atomicOr(&A.ctl->err, err);
#endif
  }
  if (!ok) return;
  if (A.cfl_next) {
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
template <int TX, int TY, int ZC, int MINB>
__global__ void __launch_bounds__(TX / 2 * TY, MINB) k_fused_pair(FusedArgs<float> A,
                                                                   const __grid_constant__ CUtensorMap map) {
  extern __shared__ __align__(128) unsigned char smem_staged[];
  auto& sm = *reinterpret_cast<PairSmem<float, TX, TY>*>(smem_staged);
  pair_tile<float, TX, TY, ZC>(A, map, sm, threadIdx.x, blockIdx.x, blockIdx.y, blockIdx.z);
}
#endif

}  // namespace EVORA_FNS
}  // namespace evora
