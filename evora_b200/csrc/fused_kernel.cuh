// fused_kernel.cuh -- the whole hydro update of one step in one HBM pass.
//
// The reference computes primitives w, ghost cells, slopes s and the
// half-step predictor evo into full-grid arrays, then sweeps x, y and z
// (muscl.f90:26-290).  All three sweeps read the same start-of-step w, s and
// evo and only add flux differences to q, in the order x, y, z per cell, so
// the update of a cell is a pure function of the start-of-step state in a
// radius-2 neighbourhood.  This kernel computes it tile by tile without
// writing any intermediate to HBM:
//
//   CTA tile = TX x TY columns (x, y) marching over ZC planes in z.
//   Per plane c:
//     A  load q of plane c+1 over the tile plus a 2-cell halo, map ghost
//        cells onto interior cells (periodic / zero-gradient mirror /
//        reflecting upper x, boundary.f90:26-113), convert to primitives
//        (q2w, comp.f90:26-85) into a 3-plane shared-memory ring;
//     B  slopes in x, y, z (comp_slope, muscl.f90:115-169) and the predictor
//        evo (muscl.f90:89-111) for the tile cells and the one-cell x/y ring,
//        then the face states w -+ s/2 + evo (muscl.f90:208-209);
//     C  one Riemann solve per x and y interface of the plane (riemann.f90)
//        into shared memory, and per column the z interface c-1/2 in
//        registers;
//     D  per owned cell: q + dt/dx (Fx- - Fx+), then + dt/dy (Fy- - Fy+)
//        (integration, muscl.f90:276-290); the z term of plane c-1 is added
//        once the flux c-1/2 is known, and plane c-1 is written out.
//
// Ghost cells are never materialised: the boundary condition is an index
// map applied when the halo is loaded.  The ping-pong output buffer keeps
// neighbouring tiles reading the start-of-step state.
//
// The same source compiles for a host emulation (EVORA_HOST_EMU) in which the
// threads of a CTA are std::threads meeting at a std::barrier, so the tile
// logic can be checked against the CPU oracle without a GPU.
#pragma once

#include "hydro_math.cuh"

#ifdef EVORA_HOST_EMU
#include <algorithm>
#include <atomic>
#include <barrier>
namespace evora_emu {
extern thread_local std::barrier<>* tl_barrier;
}
#define EV_SYNC() ::evora_emu::tl_barrier->arrive_and_wait()
#define EV_RESTRICT
#else
#define EV_SYNC() __syncthreads()
#define EV_RESTRICT __restrict__
#endif

#ifndef EVORA_FNS
#error "define EVORA_FNS (namespace of this instantiation) before including fused_kernel.cuh"
#endif

namespace evora {
namespace EVORA_FNS {

template <typename T>
struct FusedArgs {
  HydroParams P;
  const T* qin;     // NF planes of n cells, x fastest (SoA)
  T* qout;
  GridCtl* ctl;     // dt, active flag, error mask
  int64_t n;        // cells per field
  int cfl_next = 0; // 1: reduce the next step's CFL maxima into ctl->snext
  int zc = 0;       // planes per CTA (0: the instantiation's ZC)
};

// Boundary index map of one axis (0-based), boundary.f90:26-113: g in
// [-2, n+1] maps onto the interior.  Periodic wraps; zero gradient mirrors
// (ghost -1 <- cell 0, ghost -2 <- cell 1); boundtype 3 mirrors with all
// velocity components negated at the upper x face.
__device__ __forceinline__ int ghost_map(int g, int n, int bt, int axis, bool& flip) {
  if (g >= 0 && g < n) return g;
  if (bt == 2) return g < 0 ? g + n : g - n;
  if (g < 0) return -g - 1;
  if (bt == 3 && axis == 0) flip = true;
  return 2 * n - g - 1;
}

template <typename T>
__device__ __forceinline__ T ld(const T* p) {
#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
  return __ldg(p);
#else
  return *p;
#endif
}

// Primitive variables from conserved ones.  For FP64 this is q2w itself.
// For FP32 state the pressure p = (g-1)(E - kin) is recovered in FP64 when
// kin > E/2, where FP32 cancellation would lose more than one bit; with dual
// energy pressure() (comp.f90:45-85) runs with kin, the kin/E switch, E - kin
// and the resynchronised E in FP64, and rho^(g-1) in FP32 (the entropy
// branch has no cancellation; S is an FP32 field), its write-back rounded to
// FP32 (q holds 6 fields then).  The FP64 quotients are products with the
// branch-free reciprocal (rcp_fast): an FP64 division's slow-path branch
// made the FP32 dual-energy update 13 % slower.
template <typename T>
__device__ __forceinline__ void prim(T* q, T* w, const Gas<T>& c, const HydroParams& P, bool de,
                                     unsigned& err) {
  if constexpr (sizeof(T) == 8) {
    q2w(q, w, c, de, err);
  } else {
    if (de) {
      const double m2 = ((double)q[1] * q[1] + (double)q[2] * q[2]) + (double)q[3] * q[3];
      const double kin = 0.5 * m2 * rcp_fast((double)q[0]);
      const double rg = (double)powf(q[0], c.g1);
      double pd;
      if (kin * rcp_fast((double)q[4]) > P.de_thresh1) {      // S system
        pd = (double)q[5] * rg;
        q[4] = (T)(kin + pd * P.g1inv);
      } else {                                       // E system
        pd = P.g1 * ((double)q[4] - kin);
        q[5] = (T)(pd * rcp_fast(rg));
      }
      if (pd <= 0.0) err |= EVORA_ERR_PRESSURE;
      const T densinv = (T)1.0 / q[0];
      w[0] = q[0];
      w[1] = q[1] * densinv;
      w[2] = q[2] * densinv;
      w[3] = q[3] * densinv;
      w[4] = (T)pd;
      return;
    }
    T densinv = (T)1.0 / q[0];
    w[0] = q[0];
    w[1] = q[1] * densinv;
    w[2] = q[2] * densinv;
    w[3] = q[3] * densinv;
    T m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
    T kin = (T)0.5 * m2 / q[0];
    T press;
    if (kin > (T)0.5 * q[4]) {
      double dm2 = ((double)q[1] * q[1]) + ((double)q[2] * q[2]) + ((double)q[3] * q[3]);
      double dkin = 0.5 * dm2 * rcp_fast((double)q[0]);
      press = (T)(P.g1 * ((double)q[4] - dkin));
    } else {
      press = c.g1 * (q[4] - kin);
    }
    if (press <= (T)0) err |= EVORA_ERR_PRESSURE;
    w[4] = press;
  }
}

// Arithmetic form of this translation unit: EVORA_FAST = 1 selects the fast
// forms of hydro_math.cuh (FP32, default FP64), 0 the literal reference
// forms (strict FP64, and the host emulation).
#ifndef EVORA_FAST
#define EVORA_FAST 0
#endif
constexpr bool kFast = EVORA_FAST != 0;
#if defined(EVORA_HOST_EMU)
constexpr bool kHostEmu = true;    // the host emulation runs both march schedules in FP64
#else
constexpr bool kHostEmu = false;
#endif

template <typename T>
__device__ __forceinline__ T slope_k(T wl, T w, T wr, int limiter) {
  if constexpr (kFast) return slope_fast(wl, w, wr, limiter);
  else return slope1(wl, w, wr, limiter);
}

template <typename T>
__device__ __forceinline__ void pred_k(const T* w, const T* s, int d, T g, T rinv, T* a) {
  if constexpr (kFast) predictor_term_fast(w, s, d, g, rinv, a);
  else predictor_term(w, s, d, g, a);
}

template <typename T, int NF, int DIR>
__device__ __forceinline__ void riemann_k(const T* wl, const T* wr, T* f, int solver, const Gas<T>& c,
                                          unsigned& err) {
  if constexpr (kFast) riemann_fast<T, NF, DIR>(wl, wr, f, solver, c, err);
  else riemann<T, NF>(wl, wr, f, DIR, solver, c, err);
}

template <typename T>
__device__ __forceinline__ void prim_k(T* q, T* w, const Gas<T>& c, const HydroParams& P, bool de, unsigned& err) {
  if constexpr (kFast && sizeof(T) == 8) {
    if (de) q2w_de_fast(q, w, c, err);
    else q2w_fast(q, w, c, err);
    return;
  }
  prim(q, w, c, P, de, err);
}

// Shared-memory layout of one CTA (all arrays field-major).  DQ: the
// pipelined march's staging of the owned cells' state (FP32 state, FP64
// tiles that run the pipelined march, and the host emulation).
template <typename T, int NF, int TX, int TY, bool DQ = (sizeof(T) == 4 || kHostEmu)>
struct FusedSmem {
  static constexpr int RX = TX + 4, RY = TY + 4;
  T w[3][5][RY][RX];          // primitive ring: planes c-1, c, c+1 (+ halo 2)
  T xf[2][5][TY][TX + 2];     // x face states of the tile + x ring: [0] lower, [1] upper
  T yf[2][5][TY + 2][TX];     // y face states of the tile + y ring
  T fx[NF][TY][TX + 1];       // x fluxes, interface i-1/2 at column i
  T fy[NF][TY + 1][TX];       // y fluxes, interface j-1/2 at row j
  // maxima of |u_d| + a of the written cells: per thread for FP32 state
  // (whose register budget is tight), per warp otherwise
  T cfl[3][sizeof(T) == 4 ? TX * TY : 32];
  // pipelined march: the owned cells' conserved state of the plane being
  // updated, copied asynchronously one interval ahead of its use
  T dq[NF][DQ ? TX * TY : 1];
};

// Whether the shared-memory layout of a march carries dq.
template <typename T, bool PIPE>
constexpr bool kSmemDq = PIPE || sizeof(T) == 4 || kHostEmu;

// Asynchronous 4- or 8-byte global -> shared copy (cp.async), its commit
// and wait.
template <typename T>
__device__ __forceinline__ void copy_async(T* dst, const T* src) {
#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte copies");
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
#else
  *dst = *src;
#endif
}
__device__ __forceinline__ void copy_async_commit() {
#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
  asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
__device__ __forceinline__ void copy_async_wait() {
#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
  asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}

// hydrostep per cell (timestep.f90:40-43): the signal speeds |u_d| + a of
// a conserved state, in the working precision.  FP64: q2w and a = sqrt(g p
// / rho) (in the fast forms: q2w_fast or q2w_de_fast, the reciprocal and
// square root of the fast forms).  FP32 form: its primitives (FP64 pressure recovery where kin >
// E/2) and a in FP32; the maxima over cells and dt are formed in FP64 from
// these exactly representable values.  The CFL kernel and the fused
// update's reduction for the next step both call this, so either gives the
// same dt.
template <typename T, int NF>
__device__ __forceinline__ void cfl_speeds(const T* qs, const HydroParams& P, bool de, unsigned& err, T s[3]) {
  T q[6], w[5];
#pragma unroll
  for (int f = 0; f < NF; ++f) q[f] = qs[f];
  T a;
  if constexpr (sizeof(T) == 8) {
    if (kFast) {
      if (de) q2w_de_fast(q, w, Gas<double>::make(P), err);
      else q2w_fast(q, w, Gas<double>::make(P), err);
      a = sqrt_fast(P.g * w[4] * rcp_fast(w[0]));
    } else {
      q2w(q, w, Gas<double>::make(P), de, err);
      a = sqrt(P.g * w[4] / w[0]);
    }
  } else {
    prim(q, w, Gas<float>::make(P), P, de, err);
    a = sqrtf((float)P.g * w[4] / w[0]);
  }
  s[0] = fabs(w[1]) + a;
  s[1] = fabs(w[2]) + a;
  s[2] = fabs(w[3]) + a;
}

// Slopes, predictor and face states of one cell.  get(f, dx, dy, dz) reads
// primitive f of the neighbour at offset (dx, dy, dz) (one axis at a time).
// DIM = 2 or 3 selects the 2D (muscl.f90:70-88) or 3D (89-111) predictor.
template <typename T, int DIM, typename Get>
__device__ __forceinline__ void cell_faces_g(Get get, const HydroParams& P, T dt2, T* wv, T (*face)[2][5]) {
  T sx[5], sy[5], sz[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    wv[f] = get(f, 0, 0, 0);
    sx[f] = slope_k(get(f, -1, 0, 0), wv[f], get(f, 1, 0, 0), P.limiter);
    sy[f] = slope_k(get(f, 0, -1, 0), wv[f], get(f, 0, 1, 0), P.limiter);
    if (DIM == 3) sz[f] = slope_k(get(f, 0, 0, -1), wv[f], get(f, 0, 0, 1), P.limiter);
  }
  if (!P.secondorder) {
    // first-order Godunov: the face states are the cell averages (sweep,
    // muscl.f90:198-201, 207-210)
#pragma unroll
    for (int f = 0; f < 5; ++f)
#pragma unroll
      for (int d = 0; d < 3; ++d) face[d][0][f] = face[d][1][f] = wv[f];
    return;
  }
  T a1[5], a2[5], a3[5], evo[5];
  const T g = (T)P.g;
  const T rinv = kFast ? rcp_fast(wv[0]) : (T)0;
  pred_k(wv, sx, 1, g, rinv, a1);
  pred_k(wv, sy, 2, g, rinv, a2);
  if (DIM == 3) pred_k(wv, sz, 3, g, rinv, a3);
  const T dxi = (T)P.dxinv, dyi = (T)P.dyinv, dzi = (T)P.dzinv;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    if (DIM == 3) evo[f] = dt2 * (a1[f] * dxi + a2[f] * dyi + a3[f] * dzi);
    else evo[f] = dt2 * (a1[f] * dxi + a2[f] * dyi);
  }
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    face[0][0][f] = face_minus(wv[f], sx[f], evo[f]);
    face[0][1][f] = face_plus(wv[f], sx[f], evo[f]);
    face[1][0][f] = face_minus(wv[f], sy[f], evo[f]);
    face[1][1][f] = face_plus(wv[f], sy[f], evo[f]);
    if (DIM == 3) {
      face[2][0][f] = face_minus(wv[f], sz[f], evo[f]);
      face[2][1][f] = face_plus(wv[f], sz[f], evo[f]);
    }
  }
}

// cell_faces_g on the shared-memory ring: (cx, cy) are coordinates in the
// halo ring arrays, sp / sc / sn the ring slots of planes c-1, c, c+1.
template <typename T, int DIM, int TX, int TY, typename Sm>
__device__ __forceinline__ void cell_faces(const Sm& sm, int sp, int sc, int sn, int cx, int cy,
                                           const HydroParams& P, T dt2, T* wv, T (*face)[2][5]) {
  cell_faces_g<T, DIM>(
      [&](int f, int dx, int dy, int dz) -> T {
        if (dz < 0) return sm.w[sp][f][cy][cx];
        if (dz > 0) return sm.w[sn][f][cy][cx];
        return sm.w[sc][f][cy + dy][cx + dx];
      },
      P, dt2, wv, face);
}

// The tile program of one CTA.  tid in [0, TX*TY); (bx, by, bz) its tile.
// PIPE: the 3D march as a two-barrier software pipeline (FP32 state, and
// the FP64 tile entries that select it); else the three-barrier march.
template <typename T, int NF, int DIM, int TX, int TY, int ZC, bool PIPE = (sizeof(T) == 4)>
__device__ __forceinline__ void fused_tile(const FusedArgs<T>& A, FusedSmem<T, NF, TX, TY, kSmemDq<T, PIPE>>& sm,
                                           int tid, int bx, int by, int bz) {
  constexpr int NT = TX * TY;
  constexpr int RX = TX + 4, RY = TY + 4;
  const HydroParams& P = A.P;
  const int nx = P.nx, ny = P.ny, nz = DIM == 3 ? P.nz : 1;
  const int zc = A.zc > 0 ? A.zc : ZC;
  const int X0 = bx * TX, Y0 = by * TY, Z0 = DIM == 3 ? bz * zc : 0;
  const int xe = nx - X0 < TX ? nx - X0 : TX;
  const int ye = ny - Y0 < TY ? ny - Y0 : TY;
  const int ze = DIM == 3 ? (nz - Z0 < zc ? nz - Z0 : zc) : 1;
  const int oi = tid % TX, oj = tid / TX;
  const bool owned = oi < xe && oj < ye;
  const int64_t n = A.n;
  const Gas<T> c = Gas<T>::make(P);
  const bool de = NF == 6 && P.dualenergy != 0;   // dual energy carries S (nf = 6)
  unsigned err = 0;

  if (ctl_skip(A.ctl)) {
    // Inactive step: pass the state through to the other buffer.
    if (owned)
      for (int z = Z0; z < Z0 + ze; ++z) {
        const int64_t idx = ((int64_t)z * ny + (Y0 + oj)) * nx + (X0 + oi);
#pragma unroll
        for (int f = 0; f < NF; ++f) A.qout[f * n + idx] = A.qin[f * n + idx];
      }
    return;
  }

  const double dtd = A.ctl->dt;
  const T dt2 = (T)(-0.5 * dtd);
  const T dtdx = (T)(dtd * P.dxinv), dtdy = (T)(dtd * P.dyinv), dtdz = (T)(dtd * P.dzinv);

  // The next step's hydrostep maxima (timestep.f90:26-57) over the cells
  // this tile writes, computed from the written values with the CFL kernel's
  // own per-cell function (cfl_speeds), so the grid can skip that kernel's
  // pass over HBM.  With FP32 state the running maxima live in shared memory
  // (one slot per thread) rather than in registers held across the plane
  // loop.
  constexpr bool kSlots = sizeof(T) == 4;
  unsigned cerr = 0;
  T cm0 = (T)0, cm1 = (T)0, cm2 = (T)0;
  if constexpr (kSlots)
    if (A.cfl_next) sm.cfl[0][tid] = sm.cfl[1][tid] = sm.cfl[2][tid] = (T)0;
  auto track = [&](const T* qo) {
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
  };

  // A: primitives of plane z (global index, may be a ghost plane) into slot.
  // Tiles whose x/y halo lies inside the grid need no index map in x and y
  // (block-uniform test); the plane index is mapped once per plane.
  const bool interior_xy = X0 >= 2 && X0 + TX + 2 <= nx && Y0 >= 2 && Y0 + TY + 2 <= ny;
  auto load_plane = [&](int z, int slot) {
    bool zflip = false;
    const int mz = DIM == 3 ? ghost_map(z, nz, P.boundtype, 2, zflip) : 0;
    const T* plane = A.qin + (size_t)mz * ((size_t)nx * ny);   // cell index within a field < 2^31
    for (int it = tid; it < RX * RY; it += NT) {
      const int lx = it % RX, ly = it / RX;
      int gx = X0 - 2 + lx, gy = Y0 - 2 + ly;
      bool flip = false;
      int idx;
      if (interior_xy) {
        idx = gy * nx + gx;
      } else {
        // cells past the first two ghosts of a partial tile feed no owned
        // cell; clamp them onto valid cells so they hold physical data
        gx = gx > nx + 1 ? nx + 1 : gx;
        gy = gy > ny + 1 ? ny + 1 : gy;
        const int mx = ghost_map(gx, nx, P.boundtype, 0, flip);
        const int my = ghost_map(gy, ny, P.boundtype, 1, flip);
        idx = my * nx + mx;
      }
      T qv[6], wv[5];
#pragma unroll
      for (int f = 0; f < NF; ++f) qv[f] = ld(plane + (size_t)f * n + idx);
      prim_k(qv, wv, c, P, de, err);
      if (flip) {
        wv[1] = -wv[1];
        wv[2] = -wv[2];
        wv[3] = -wv[3];
      }
#pragma unroll
      for (int f = 0; f < 5; ++f) sm.w[slot][f][ly][lx] = wv[f];
    }
  };

  // Per-column state carried across planes (registers of the owner).
  T qacc[NF];       // plane c-1 after its x and y terms
  T wzp_prev[5];    // upper z face state of plane c-1
  T fz_prev[NF];    // z flux through c-3/2
#pragma unroll
  for (int f = 0; f < NF; ++f) { qacc[f] = (T)0; fz_prev[f] = (T)0; }
#pragma unroll
  for (int f = 0; f < 5; ++f) wzp_prev[f] = (T)0;

  const int zfirst = DIM == 3 ? Z0 - 1 : 0;
  const int zlast = DIM == 3 ? Z0 + ze : 0;
  auto slot_of = [&](int z) { return (z - (Z0 - 2)) % 3; };

  if constexpr (DIM == 3 && PIPE) {
    // Software-pipelined march, two barriers per plane.  Iteration c (an
    // inner plane) runs
    //   I1: A(c+2) and the x/y Riemann solves of plane c      | barrier
    //   I2: D(c), B(c+1) and the z flux through c+1/2         | barrier
    // with B(c) and the z flux through c-1/2 done before it.  A(c+2) refills
    // the ring slot of plane c-1, last read by B(c) before the previous
    // barrier; B(c+1) rewrites face states the solves of plane c consumed
    // before the last one; C(c+1) rewrites fluxes D(c) read before it.
    T wzp_c[5];      // upper z face of the current plane
    T fz_cur[NF];    // z flux through c-1/2 (then c+1/2)
    auto faces = [&](int cz, bool in, T* wzm, T* wzp) {
      const int sp = slot_of(cz - 1), sc = slot_of(cz), sn = slot_of(cz + 1);
      if (owned) {
        T wv[5], face[3][2][5];
        cell_faces<T, DIM, TX, TY>(sm, sp, sc, sn, oi + 2, oj + 2, P, dt2, wv, face);
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
      if (in) {
        // ring cells: x ring at x = -1 and x = xe (rows 0..ye-1),
        // y ring at y = -1 and y = ye (columns 0..xe-1)
        const int nring = 2 * ye + 2 * xe;
        for (int r = tid; r < nring; r += NT) {
          int li, lj;
          bool xring;
          if (r < 2 * ye) {
            xring = true;
            lj = r >> 1;
            li = (r & 1) ? xe : -1;
          } else {
            xring = false;
            const int rr = r - 2 * ye;
            li = rr >> 1;
            lj = (rr & 1) ? ye : -1;
          }
          T wv[5], face[3][2][5];
          cell_faces<T, DIM, TX, TY>(sm, sp, sc, sn, li + 2, lj + 2, P, dt2, wv, face);
          if (xring) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
              sm.xf[0][f][lj][li + 1] = face[0][0][f];
              sm.xf[1][f][lj][li + 1] = face[0][1][f];
            }
          } else {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
              sm.yf[0][f][lj + 1][li] = face[1][0][f];
              sm.yf[1][f][lj + 1][li] = face[1][1][f];
            }
          }
        }
      }
    };
    auto solves_xy = [&]() {
      // counted from the last thread: the threads that load one halo cell
      // fewer in A take the extra solves of the same interval
      const int nxi = (xe + 1) * ye, nyi = xe * (ye + 1);
      for (int it = NT - 1 - tid; it < nxi + nyi; it += NT) {
        T wl[5], wr[5], fv[NF];
        if (it < nxi) {
          const int i = it % (xe + 1), j = it / (xe + 1);
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            wl[f] = sm.xf[1][f][j][i];
            wr[f] = sm.xf[0][f][j][i + 1];
          }
          riemann_k<T, NF, 1>(wl, wr, fv, P.solver, c, err);
#pragma unroll
          for (int f = 0; f < NF; ++f) sm.fx[f][j][i] = fv[f];
        } else {
          const int r = it - nxi;
          const int i = r % xe, j = r / xe;
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            wl[f] = sm.yf[1][f][j][i];
            wr[f] = sm.yf[0][f][j + 1][i];
          }
          riemann_k<T, NF, 2>(wl, wr, fv, P.solver, c, err);
#pragma unroll
          for (int f = 0; f < NF; ++f) sm.fy[f][j][i] = fv[f];
        }
      }
    };
    auto zflux = [&](const T* lo_plane_upper, const T* hi_plane_lower, T* fz) {
#pragma unroll
      for (int f = 0; f < NF; ++f) fz[f] = (T)0;
      if (owned) riemann_k<T, NF, 3>(lo_plane_upper, hi_plane_lower, fz, P.solver, c, err);
    };
    // plane z (held in qacc after its x and y terms) gets its z term
    auto write_plane = [&](int z, const T* fz_lo, const T* fz_hi) {
      if (!owned) return;
      const int64_t idx = ((int64_t)z * ny + (Y0 + oj)) * nx + (X0 + oi);
      T qo[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        qo[f] = qacc[f] + dtdz * (fz_lo[f] - fz_hi[f]);
        A.qout[f * n + idx] = qo[f];
      }
      if (A.cfl_next) track(qo);
    };
    // the owned cell's conserved state of plane z into sm.dq, asynchronously
    // (waited for by the same thread in update_xy, one interval later)
    auto prefetch_own = [&](int z) {
      if (!owned) return;
      const int64_t idx = ((int64_t)z * ny + (Y0 + oj)) * nx + (X0 + oi);
#pragma unroll
      for (int f = 0; f < NF; ++f) copy_async(&sm.dq[f][tid], A.qin + f * n + idx);
      copy_async_commit();
    };
    // plane z: q + the x and y flux differences, into qacc
    auto update_xy = [&](int z) {
      if (!owned) return;
      (void)z;
      copy_async_wait();
      T qv[6], wdummy[5];
#pragma unroll
      for (int f = 0; f < NF; ++f) qv[f] = sm.dq[f][tid];
      if (de) {
        unsigned e2 = 0;
        prim_k(qv, wdummy, c, P, de, e2);  // dual-energy resync of q (comp.f90:60-72)
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) qv[f] = qv[f] + dtdx * (sm.fx[f][oj][oi] - sm.fx[f][oj][oi + 1]);
#pragma unroll
      for (int f = 0; f < NF; ++f) qacc[f] = qv[f] + dtdy * (sm.fy[f][oj][oi] - sm.fy[f][oj + 1][oi]);
    };

    // prologue: planes Z0-2 .. Z0+1, B of the plane below the tile and of
    // the first plane, the z flux through Z0 - 1/2
    T wzm_n[5], wzp_n[5];
    load_plane(Z0 - 2, slot_of(Z0 - 2));
    load_plane(Z0 - 1, slot_of(Z0 - 1));
    load_plane(Z0, slot_of(Z0));
    EV_SYNC();
    faces(Z0 - 1, false, wzm_n, wzp_c);
    EV_SYNC();
    load_plane(Z0 + 1, slot_of(Z0 + 1));
    EV_SYNC();
    faces(Z0, true, wzm_n, wzp_n);
    zflux(wzp_c, wzm_n, fz_cur);
#pragma unroll
    for (int f = 0; f < 5; ++f) wzp_c[f] = wzp_n[f];
    EV_SYNC();
    for (int cz = Z0; cz < Z0 + ze; ++cz) {
      // ---- I1
      prefetch_own(cz);
      load_plane(cz + 2, slot_of(cz + 2));
      solves_xy();
      EV_SYNC();
      // ---- I2
      if (cz > Z0) write_plane(cz - 1, fz_prev, fz_cur);
      update_xy(cz);
      faces(cz + 1, cz + 1 < Z0 + ze, wzm_n, wzp_n);
#pragma unroll
      for (int f = 0; f < NF; ++f) fz_prev[f] = fz_cur[f];
      zflux(wzp_c, wzm_n, fz_cur);
#pragma unroll
      for (int f = 0; f < 5; ++f) wzp_c[f] = wzp_n[f];
      EV_SYNC();
    }
    write_plane(Z0 + ze - 1, fz_prev, fz_cur);
    (void)zfirst;
    (void)zlast;
  } else
  for (int cz = zfirst; cz <= zlast; ++cz) {
    const bool inner = cz >= Z0 && cz < Z0 + ze;  // plane cz is updated by this tile
    if (DIM == 3 && cz == zfirst) {
      // the two planes below the march
      load_plane(Z0 - 2, slot_of(Z0 - 2));
      load_plane(Z0 - 1, slot_of(Z0 - 1));
    }
    // ---- A
    if (DIM == 3) load_plane(cz + 1, slot_of(cz + 1));
    else load_plane(0, 1);
    EV_SYNC();
    const int sp = DIM == 3 ? slot_of(cz - 1) : 0;
    const int sc = DIM == 3 ? slot_of(cz) : 1;
    const int sn = DIM == 3 ? slot_of(cz + 1) : 2;
    // ---- B
    T wzm_cur[5], wzp_cur[5];
    if (owned) {
      T wv[5], face[3][2][5];
      cell_faces<T, DIM, TX, TY>(sm, sp, sc, sn, oi + 2, oj + 2, P, dt2, wv, face);
      if (inner) {
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
        wzm_cur[f] = face[2][0][f];
        wzp_cur[f] = face[2][1][f];
      }
    }
    if (inner) {
      // ring cells: x ring at x = -1 and x = xe (rows 0..ye-1),
      // y ring at y = -1 and y = ye (columns 0..xe-1)
      const int nring = 2 * ye + 2 * xe;
      for (int r = tid; r < nring; r += NT) {
        int li, lj;
        bool xring;
        if (r < 2 * ye) {
          xring = true;
          lj = r >> 1;
          li = (r & 1) ? xe : -1;
        } else {
          xring = false;
          const int rr = r - 2 * ye;
          li = rr >> 1;
          lj = (rr & 1) ? ye : -1;
        }
        T wv[5], face[3][2][5];
        cell_faces<T, DIM, TX, TY>(sm, sp, sc, sn, li + 2, lj + 2, P, dt2, wv, face);
        if (xring) {
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            sm.xf[0][f][lj][li + 1] = face[0][0][f];
            sm.xf[1][f][lj][li + 1] = face[0][1][f];
          }
        } else {
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            sm.yf[0][f][lj + 1][li] = face[1][0][f];
            sm.yf[1][f][lj + 1][li] = face[1][1][f];
          }
        }
      }
    }
    EV_SYNC();
    // ---- C
    if (inner) {
      const int nxi = (xe + 1) * ye, nyi = xe * (ye + 1);
      for (int it = tid; it < nxi + nyi; it += NT) {
        T wl[5], wr[5], fv[NF];
        if (it < nxi) {
          const int i = it % (xe + 1), j = it / (xe + 1);
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            wl[f] = sm.xf[1][f][j][i];
            wr[f] = sm.xf[0][f][j][i + 1];
          }
          riemann_k<T, NF, 1>(wl, wr, fv, P.solver, c, err);
#pragma unroll
          for (int f = 0; f < NF; ++f) sm.fx[f][j][i] = fv[f];
        } else {
          const int r = it - nxi;
          const int i = r % xe, j = r / xe;
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            wl[f] = sm.yf[1][f][j][i];
            wr[f] = sm.yf[0][f][j + 1][i];
          }
          riemann_k<T, NF, 2>(wl, wr, fv, P.solver, c, err);
#pragma unroll
          for (int f = 0; f < NF; ++f) sm.fy[f][j][i] = fv[f];
        }
      }
    }
    T fz[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) fz[f] = (T)0;
    if (DIM == 3 && owned && cz > zfirst) riemann_k<T, NF, 3>(wzp_prev, wzm_cur, fz, P.solver, c, err);
    EV_SYNC();
    // ---- D
    if (owned) {
      if (DIM == 3 && cz - 1 >= Z0 && cz - 1 < Z0 + ze) {
        // plane cz-1 gets its z term and is written out
        const int64_t idx = ((int64_t)(cz - 1) * ny + (Y0 + oj)) * nx + (X0 + oi);
        T qo[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          qo[f] = qacc[f] + dtdz * (fz_prev[f] - fz[f]);
          A.qout[f * n + idx] = qo[f];
        }
        if (A.cfl_next) track(qo);
      }
      if (inner) {
        const int64_t idx = ((int64_t)cz * ny + (Y0 + oj)) * nx + (X0 + oi);
        T qv[6], wdummy[5];
#pragma unroll
        for (int f = 0; f < NF; ++f) qv[f] = ld(A.qin + f * n + idx);
        if (de) {
          unsigned e2 = 0;
          prim_k(qv, wdummy, c, P, de, e2);  // dual-energy resync of q (comp.f90:60-72)
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) qv[f] = qv[f] + dtdx * (sm.fx[f][oj][oi] - sm.fx[f][oj][oi + 1]);
#pragma unroll
        for (int f = 0; f < NF; ++f) qv[f] = qv[f] + dtdy * (sm.fy[f][oj][oi] - sm.fy[f][oj + 1][oi]);
        if (DIM == 3) {
#pragma unroll
          for (int f = 0; f < NF; ++f) qacc[f] = qv[f];
        } else {
#pragma unroll
          for (int f = 0; f < NF; ++f) A.qout[f * n + idx] = qv[f];
          if (A.cfl_next) track(qv);
        }
      }
      if (DIM == 3) {
#pragma unroll
        for (int f = 0; f < NF; ++f) fz_prev[f] = fz[f];
#pragma unroll
        for (int f = 0; f < 5; ++f) wzp_prev[f] = wzp_cur[f];
      }
    }
  }
  if (err) {
#if defined(EVORA_HOST_EMU)
    reinterpret_cast<std::atomic<unsigned>*>(&A.ctl->err)->fetch_or(err);
#else
    atomicOr(&A.ctl->err, err);
#endif
  }
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
    EV_SYNC();   // every thread has read its own slots
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

// 1D grids: one thread per cell.  The cell rebuilds the primitives of its
// radius-2 neighbourhood, the face states of cells i-1, i, i+1 with the 1D
// predictor (muscl.f90:60-69) and solves its two interfaces.
template <typename T, int NF>
__device__ __forceinline__ void fused_cell1d(const FusedArgs<T>& A, int i) {
  const HydroParams& P = A.P;
  const int nx = P.nx;
  const int64_t n = A.n;
  if (ctl_skip(A.ctl)) {
#pragma unroll
    for (int f = 0; f < NF; ++f) A.qout[f * n + i] = A.qin[f * n + i];
    return;
  }
  const Gas<T> c = Gas<T>::make(P);
  const bool de = NF == 6 && P.dualenergy != 0;   // dual energy carries S (nf = 6)
  unsigned err = 0;
  const double dtd = A.ctl->dt;
  const T dt2 = (T)(-0.5 * dtd);
  const T dtdx = (T)(dtd * P.dxinv);
  const T dxi = (T)P.dxinv;
  T w[5][5];
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    bool flip = false;
    const int m = ghost_map(i - 2 + o, nx, P.boundtype, 0, flip);
    T qv[6];
#pragma unroll
    for (int f = 0; f < NF; ++f) qv[f] = ld(A.qin + f * n + m);
    prim_k(qv, w[o], c, P, de, err);
    if (flip) {
      w[o][1] = -w[o][1];
      w[o][2] = -w[o][2];
      w[o][3] = -w[o][3];
    }
  }
  T fm[3][5], fp[3][5];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (P.secondorder) {
      T s[5], a[5];
#pragma unroll
      for (int f = 0; f < 5; ++f) s[f] = slope_k(w[k][f], w[k + 1][f], w[k + 2][f], P.limiter);
      pred_k(w[k + 1], s, 1, (T)P.g, kFast ? rcp_fast(w[k + 1][0]) : (T)0, a);
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        const T e = dt2 * a[f] * dxi;
        fm[k][f] = face_minus(w[k + 1][f], s[f], e);
        fp[k][f] = face_plus(w[k + 1][f], s[f], e);
      }
    } else {
#pragma unroll
      for (int f = 0; f < 5; ++f) fm[k][f] = fp[k][f] = w[k + 1][f];
    }
  }
  T flo[NF], fhi[NF];
  riemann_k<T, NF, 1>(fp[0], fm[1], flo, P.solver, c, err);
  riemann_k<T, NF, 1>(fp[1], fm[2], fhi, P.solver, c, err);
  T qv[6], wd[5];
#pragma unroll
  for (int f = 0; f < NF; ++f) qv[f] = ld(A.qin + f * n + i);
  if (de) {
    unsigned e2 = 0;
    prim_k(qv, wd, c, P, de, e2);
  }
#pragma unroll
  for (int f = 0; f < NF; ++f) A.qout[f * n + i] = qv[f] + dtdx * (flo[f] - fhi[f]);
  if (err) {
#if defined(EVORA_HOST_EMU)
    reinterpret_cast<std::atomic<unsigned>*>(&A.ctl->err)->fetch_or(err);
#else
    atomicOr(&A.ctl->err, err);
#endif
  }
}

#if !defined(EVORA_HOST_EMU)
template <typename T, int NF>
__global__ void __launch_bounds__(128) k_fused1d(FusedArgs<T> A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.P.nx; i += gridDim.x * blockDim.x)
    fused_cell1d<T, NF>(A, i);
}

// MINB: CTAs per SM the register allocation must allow (shared memory is
// sized for the same count; see the tile table in fused_inst.cuh).  PIPE:
// the march (fused_tile).
template <typename T, int NF, int DIM, int TX, int TY, int ZC, int MINB, bool PIPE = (sizeof(T) == 4)>
__global__ void __launch_bounds__(TX* TY, MINB) k_fused(FusedArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto& sm = *reinterpret_cast<FusedSmem<T, NF, TX, TY, kSmemDq<T, PIPE>>*>(smem_raw);
  fused_tile<T, NF, DIM, TX, TY, ZC, PIPE>(A, sm, threadIdx.x, blockIdx.x, blockIdx.y, blockIdx.z);
}
#endif

}  // namespace EVORA_FNS
}  // namespace evora
