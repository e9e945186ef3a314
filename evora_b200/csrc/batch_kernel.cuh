// batch_kernel.cuh -- many independent 1D tubes advanced in one persistent
// launch.
//
// Each tube is a 1D grid of its own length with its own time t, step size dt
// and end time (the hydro loop main.f90:109-155 per tube: primitive, bound,
// hydrostep, updatetime, compevo, sweep with the 1D predictor of
// muscl.f90:60-69).  A CTA pulls the next tube from a work queue (tubes are
// ordered by estimated work, largest first), stages its conserved state in
// shared memory and runs up to `budget` steps of that tube without leaving
// the SM, then writes the state back: HBM sees each tube once per launch.
//
// Per step, with the tube in shared memory:
//   phase 1  primitives of the n cells and the 2+2 ghost cells (index map of
//            bound, boundary.f90:33-66) into w; per-thread maxima of
//            |u_d| + a; block reduction; thread 0 forms dt (hydrostep) and
//            advances t (updatetime);
//   phase 2  every thread sweeps a contiguous segment of cells like the
//            reference's pencil loop (muscl.f90:194-215): face states from
//            the slopes and the predictor, one Riemann solve per interface,
//            the flux of the previous interface carried, q updated in place.
// A tube longer than the shared-memory capacity keeps q in a global scratch
// slot of its CTA and w in shared memory while w alone fits, else both in
// the slot (same code, generic pointers).
#pragma once

#include "batch.h"
#include "fused_kernel.cuh"

namespace evora {
namespace EVORA_FNS {

template <typename T, int NF, int NT>
__device__ __forceinline__ void tube_run(const BatchArgs<T>& A, T* qs, T* w, int tb, double* red,
                                         double* bc, unsigned* s_err) {
  const int tid = threadIdx.x;
  TubeState* ts = A.tubes + tb;
  const int n = ts->n;
  const long long off = ts->offset;
  const HydroParams& PP = A.P;
  // compparameter for this tube (parameter.f90:192-205, 1D branch)
  HydroParams P = PP;
  if (ts->bt) P.boundtype = ts->bt;
  P.nx = n;
  P.ny = 1;
  P.nz = 1;
  P.dx = (A.xmax - A.xmin) / n;
  P.dy = P.dx;
  P.dz = P.dx;
  {
    double ymax = P.dy, zmax = P.dz;
    P.dy = (ymax - 0.0) / 1;
    P.dz = (zmax - 0.0) / 1;
  }
  P.dxinv = 1.0 / P.dx;
  P.dyinv = 1.0 / P.dy;
  P.dzinv = 1.0 / P.dz;
  const Gas<T> c = Gas<T>::make(P);
  const bool de = P.dualenergy != 0;
  const int wst = n + 4;        // w row stride (2 ghosts each side)
  // stage q into qs (field-major, stride n)
  for (int f = 0; f < NF; ++f)
    for (int i = tid; i < n; i += NT) qs[f * n + i] = A.q[(size_t)f * A.ntot + off + i];
  double t = ts->t, dt = ts->dt, tend = ts->tend;
  unsigned err = 0;
  int steps = 0, go = 1;
  if (tid == 0) *s_err = 0u;
  int budget = A.budget;
  if (A.quantum > 0) {
    const long long b = A.quantum / n;
    budget = (int)(b < 1 ? 1 : (b < budget ? b : budget));
  }
  __syncthreads();
  while (steps < budget) {
    // ---- phase 1: primitives (+ ghosts) and the CFL maxima
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (int i = tid; i < wst; i += NT) {
      bool flip = false;
      const int g = ghost_map(i - 2, n, P.boundtype, 0, flip);
      T qv[6], wv[5];
#pragma unroll
      for (int f = 0; f < NF; ++f) qv[f] = qs[f * n + g];
      prim_k(qv, wv, c, P, de, err);
      if (flip) {
        wv[1] = -wv[1];
        wv[2] = -wv[2];
        wv[3] = -wv[3];
      }
#pragma unroll
      for (int f = 0; f < 5; ++f) w[f * wst + i] = wv[f];
      if (i >= 2 && i < n + 2) {
        // hydrostep speeds (timestep.f90:40-43), reduced in FP64
        const T a = dsqrt(c.g * wv[4] / wv[0]);
        const double s0 = (double)(fabs(wv[1]) + a), s1 = (double)(fabs(wv[2]) + a),
                     s2 = (double)(fabs(wv[3]) + a);
        if (s0 > m0) m0 = s0;
        if (s1 > m1) m1 = s1;
        if (s2 > m2) m2 = s2;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      m0 = fmax2(m0, __shfl_xor_sync(0xffffffffu, m0, o));
      m1 = fmax2(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmax2(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) {
      red[3 * wid + 0] = m0;
      red[3 * wid + 1] = m1;
      red[3 * wid + 2] = m2;
    }
    if (err) atomicOr(s_err, err);
    __syncthreads();
    if (tid == 0) {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int k = 0; k < NT / 32; ++k) {
        a0 = fmax2(a0, red[3 * k]);
        a1 = fmax2(a1, red[3 * k + 1]);
        a2 = fmax2(a2, red[3 * k + 2]);
      }
      unsigned e = *s_err;
      double d = cfl_dt(P, a0, a1, a2, 1e99, e);
      int g2 = 1;
      double tt = t;
      if (!e) update_time(tend, tt, d, g2);
      if (!e && g2 && !(tt > t)) e |= EVORA_ERR_DT;   // dt below the resolution of t: no progress
      bc[0] = d;
      bc[1] = tt;
      bc[2] = e ? 1.0 : 0.0;
      bc[3] = g2;
      *s_err = e;
    }
    __syncthreads();
    if (bc[2] != 0.0) break;       // an error stops the tube before its update
    dt = bc[0];
    t = bc[1];
    go = (int)bc[3];
    // ---- phase 2: segment sweeps
    const T dt2 = (T)(-0.5 * dt);
    const T dtdx = (T)(dt * P.dxinv);
    const T dxi = (T)P.dxinv;
    const int seg = (n + NT - 1) / NT;
    const int i0 = tid * seg;
    const int i1 = i0 + seg < n ? i0 + seg : n;
    if (i0 < i1) {
      T fp_prev[5], flo[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) flo[f] = (T)0;
      for (int cc = i0 - 1; cc <= i1; ++cc) {
        const int wi = cc + 2;
        T wc[5], fm[5], fp[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) wc[f] = w[f * wst + wi];
        if (P.secondorder) {
          T s[5], a[5];
#pragma unroll
          for (int f = 0; f < 5; ++f) s[f] = slope_k(w[f * wst + wi - 1], wc[f], w[f * wst + wi + 1], P.limiter);
          pred_k(wc, s, 1, c.g, kFast ? rcp_fast(wc[0]) : (T)0, a);
#pragma unroll
          for (int f = 0; f < 5; ++f) {
            const T e = dt2 * a[f] * dxi;                  // muscl.f90:68
            fm[f] = face_minus(wc[f], s[f], e);
            fp[f] = face_plus(wc[f], s[f], e);
          }
        } else {
#pragma unroll
          for (int f = 0; f < 5; ++f) fm[f] = fp[f] = wc[f];
        }
        if (cc > i0 - 1) {
          T fr[NF];
          riemann_k<T, NF, 1>(fp_prev, fm, fr, P.solver, c, err);   // interface cc-1/2
          if (cc - 1 >= i0) {
            T qv[6], wd[5];
#pragma unroll
            for (int f = 0; f < NF; ++f) qv[f] = qs[f * n + cc - 1];
            if (de) {
              unsigned e2 = 0;
              prim_k(qv, wd, c, P, de, e2);
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) qs[f * n + cc - 1] = qv[f] + dtdx * (flo[f] - fr[f]);
          }
#pragma unroll
          for (int f = 0; f < NF; ++f) flo[f] = fr[f];
        }
#pragma unroll
        for (int f = 0; f < 5; ++f) fp_prev[f] = fp[f];
      }
    }
    ++steps;
    if (err) atomicOr(s_err, err);
    __syncthreads();
    if (!go || *s_err) break;     // a Riemann error stops the tube after its step
  }
  // write back
  for (int f = 0; f < NF; ++f)
    for (int i = tid; i < n; i += NT) A.q[(size_t)f * A.ntot + off + i] = qs[f * n + i];
  __syncthreads();
  if (tid == 0) {
    const unsigned e = *s_err;
    ts->err |= e;
    ts->t = t;
    ts->dt = dt;
    ts->k += steps;
    if (e) ts->status = TUBE_ERROR;
    else if (!go) ts->status = TUBE_DONE;
    atomicAdd((unsigned long long*)A.cell_updates, (unsigned long long)n * (unsigned long long)steps);
  }
}

template <typename T, int NF, int NT>
__global__ void __launch_bounds__(NT) k_tubes(BatchArgs<T> A) {
  extern __shared__ __align__(16) unsigned char sraw[];
  __shared__ int s_tube;
  __shared__ double red[3 * (NT / 32)];
  __shared__ double bc[4];
  __shared__ unsigned s_err;
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = atomicAdd(A.head, 1);
      s_tube = i < A.ntubes ? A.order[i] : -1;
    }
    __syncthreads();
    const int tb = s_tube;
    __syncthreads();
    if (tb < 0) break;
    if (A.tubes[tb].status != TUBE_RUNNING) continue;
    const int n = A.tubes[tb].n;
    T* qs;
    T* w;
    if (n <= A.cap) {
      qs = reinterpret_cast<T*>(sraw);
      w = qs + NF * A.cap;
    } else if (n <= A.capw) {
      // the primitives (read three times per cell and step by the sweeps)
      // in shared memory, the state in the CTA's scratch slot
      w = reinterpret_cast<T*>(sraw);
      qs = A.gscratch + (size_t)blockIdx.x * (size_t)(NF + 5) * (A.nmax + 4);
    } else {
      qs = A.gscratch + (size_t)blockIdx.x * (size_t)(NF + 5) * (A.nmax + 4);
      w = qs + (size_t)NF * (A.nmax + 4);
    }
    tube_run<T, NF, NT>(A, qs, w, tb, red, bc, &s_err);
  }
}

}  // namespace EVORA_FNS
}  // namespace evora
