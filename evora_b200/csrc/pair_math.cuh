// pair_math.cuh -- per-cell hydro arithmetic on two cells at once.
//
// P2<S> holds one value of two cells.  On the device with S = float, every
// add, subtract, multiply and fused multiply-add of a pair is one packed
// sm_100 instruction (add/sub/mul/fma .rn.ftz.f32x2); comparisons, selects,
// min/max, reciprocals and square roots act per cell.  The formulas are the
// fast forms of hydro_math.cuh (FP32 form): q2w with one reciprocal and the
// FP64 pressure recovery where kin > E/2 (comp.f90:26-85), the minmod
// limiter (muscl.f90:128-140, written as the median of 0 and the two
// differences), the 3D predictor (muscl.f90:89-111), the face states
// (muscl.f90:199-209) and HLLC (riemann.f90:96-205, with the sl = 0 / sr = 0
// gap closed as in hllc_fast).  The association of sums may differ from the
// scalar FP32 form (results agree to FP32 rounding); the host build (S =
// double, plain operators) is used by the emulation test harness.
#pragma once

#include "hydro_math.cuh"

namespace evora {

template <typename S>
struct P2 {
  S x, y;
};

template <typename S>
__device__ __forceinline__ P2<S> p2(S v) { return P2<S>{v, v}; }

#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
__device__ __forceinline__ unsigned long long pk(P2<float> a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ P2<float> upk(unsigned long long r) {
  P2<float> a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ P2<float> operator+(P2<float> a, P2<float> b) {
  unsigned long long r;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
  return upk(r);
}
__device__ __forceinline__ P2<float> operator-(P2<float> a, P2<float> b) {
  unsigned long long r;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
  return upk(r);
}
__device__ __forceinline__ P2<float> operator*(P2<float> a, P2<float> b) {
  unsigned long long r;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
  return upk(r);
}
// a * b + c
__device__ __forceinline__ P2<float> fma2(P2<float> a, P2<float> b, P2<float> c) {
  unsigned long long r;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
  return upk(r);
}
#endif

// Generic (host emulation, and FP64 pairs): per component.
template <typename S>
__device__ __forceinline__ P2<S> operator+(P2<S> a, P2<S> b) { return P2<S>{a.x + b.x, a.y + b.y}; }
template <typename S>
__device__ __forceinline__ P2<S> operator-(P2<S> a, P2<S> b) { return P2<S>{a.x - b.x, a.y - b.y}; }
template <typename S>
__device__ __forceinline__ P2<S> operator*(P2<S> a, P2<S> b) { return P2<S>{a.x * b.x, a.y * b.y}; }
template <typename S>
__device__ __forceinline__ P2<S> fma2(P2<S> a, P2<S> b, P2<S> c) { return P2<S>{a.x * b.x + c.x, a.y * b.y + c.y}; }

template <typename S>
__device__ __forceinline__ P2<S> neg2(P2<S> a) { return P2<S>{-a.x, -a.y}; }
template <typename S>
__device__ __forceinline__ P2<S> min2(P2<S> a, P2<S> b) { return P2<S>{fmin2(a.x, b.x), fmin2(a.y, b.y)}; }
template <typename S>
__device__ __forceinline__ P2<S> max2(P2<S> a, P2<S> b) { return P2<S>{fmax2(a.x, b.x), fmax2(a.y, b.y)}; }
template <typename S>
__device__ __forceinline__ P2<S> abs2(P2<S> a) { return P2<S>{fabs(a.x), fabs(a.y)}; }
template <typename S>
__device__ __forceinline__ P2<S> rcp2(P2<S> a) { return P2<S>{rcp_fast(a.x), rcp_fast(a.y)}; }
template <typename S>
__device__ __forceinline__ P2<S> sqrt2(P2<S> a) { return P2<S>{dsqrt(a.x), dsqrt(a.y)}; }

struct M2 {
  bool x, y;
};
template <typename S>
__device__ __forceinline__ P2<S> sel2(M2 m, P2<S> a, P2<S> b) { return P2<S>{m.x ? a.x : b.x, m.y ? a.y : b.y}; }

// q2w of two cells (comp.f90:26-85 without dual energy), FP32 form: FP32
// arithmetic with the pressure recovered in FP64 for a cell whose kinetic
// energy exceeds half its total energy.
template <typename S>
__device__ __forceinline__ void prim_p(const P2<S>* q, P2<S>* w, const Gas<S>& c, const HydroParams& P,
                                       unsigned& err) {
  const P2<S> densinv = rcp2(q[0]);
  w[0] = q[0];
  w[1] = q[1] * densinv;
  w[2] = q[2] * densinv;
  w[3] = q[3] * densinv;
  const P2<S> m2 = fma2(q[3], q[3], fma2(q[2], q[2], q[1] * q[1]));
  const P2<S> kin = (p2<S>((S)0.5) * m2) * densinv;
  P2<S> press = p2<S>(c.g1) * (q[4] - kin);
  if constexpr (sizeof(S) == 4) {
    const bool hx = kin.x > (S)0.5 * q[4].x, hy = kin.y > (S)0.5 * q[4].y;
    if (hx || hy) {
      auto rec = [&](S q0, S q1, S q2, S q3, S q4) -> S {
        const double dm2 = ((double)q1 * q1) + ((double)q2 * q2) + ((double)q3 * q3);
        return (S)(P.g1 * ((double)q4 - 0.5 * dm2 * rcp_fast((double)q0)));
      };
      if (hx) press.x = rec(q[0].x, q[1].x, q[2].x, q[3].x, q[4].x);
      if (hy) press.y = rec(q[0].y, q[1].y, q[2].y, q[3].y, q[4].y);
    }
  }
  if (press.x <= (S)0 || press.y <= (S)0) err |= EVORA_ERR_PRESSURE;
  w[4] = press;
}

// minmod(w - wl, wr - w) (muscl.f90:128-140) as median(0, a, b).
template <typename S>
__device__ __forceinline__ P2<S> minmod_p(P2<S> wl, P2<S> w, P2<S> wr) {
  const P2<S> a = w - wl, b = wr - w;
  const P2<S> z = p2<S>((S)0);
  return max2(min2(a, b), min2(max2(a, b), z));
}

// Slopes, 3D predictor and the six face states of two cells.  get(f, dx,
// dy, dz) reads primitive f of the neighbour pair at offset (dx, dy, dz).
// face[d][0] is the lower and face[d][1] the upper face of axis d.
template <typename S, typename Get>
__device__ __forceinline__ void faces_p(Get get, const HydroParams& P, S dt2, P2<S>* wv, P2<S> (*face)[2][5]) {
  P2<S> sx[5], sy[5], sz[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    wv[f] = get(f, 0, 0, 0);
    sx[f] = minmod_p(get(f, -1, 0, 0), wv[f], get(f, 1, 0, 0));
    sy[f] = minmod_p(get(f, 0, -1, 0), wv[f], get(f, 0, 1, 0));
    sz[f] = minmod_p(get(f, 0, 0, -1), wv[f], get(f, 0, 0, 1));
  }
  // predictor (muscl.f90:100-104): a_d(f) = u_d s_d(f), + g p s_d(u_d) on
  // the pressure row, + s_d(p) / rho on the u_d row
  const P2<S> rinv = rcp2(wv[0]);
  const P2<S> gp = p2<S>((S)P.g) * wv[4];
  P2<S> evo[5];
  const P2<S> cx = p2<S>(dt2 * (S)P.dxinv), cy = p2<S>(dt2 * (S)P.dyinv), cz = p2<S>(dt2 * (S)P.dzinv);
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    P2<S> ax = wv[1] * sx[f], ay = wv[2] * sy[f], az = wv[3] * sz[f];
    if (f == 4) {
      ax = fma2(gp, sx[1], ax);
      ay = fma2(gp, sy[2], ay);
      az = fma2(gp, sz[3], az);
    }
    if (f == 1) ax = fma2(sx[4], rinv, ax);
    if (f == 2) ay = fma2(sy[4], rinv, ay);
    if (f == 3) az = fma2(sz[4], rinv, az);
    evo[f] = fma2(cz, az, fma2(cy, ay, cx * ax));
  }
  const P2<S> h = p2<S>((S)0.5), mh = p2<S>((S)-0.5);
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const P2<S> t = wv[f] + evo[f];
    face[0][0][f] = fma2(mh, sx[f], t);
    face[0][1][f] = fma2(h, sx[f], t);
    face[1][0][f] = fma2(mh, sy[f], t);
    face[1][1][f] = fma2(h, sy[f], t);
    face[2][0][f] = fma2(mh, sz[f], t);
    face[2][1][f] = fma2(h, sz[f], t);
  }
}

// HLLC flux of two interfaces along axis DIR (1..3), fast form.
template <typename S, int DIR>
__device__ __forceinline__ void hllc_p(const P2<S>* wl, const P2<S>* wr, P2<S>* f, const Gas<S>& c,
                                       unsigned& err) {
  if (wl[4].x <= (S)0 || wl[4].y <= (S)0 || wr[4].x <= (S)0 || wr[4].y <= (S)0) err |= EVORA_ERR_RIEMANN_PRESSURE;
  const P2<S> ril = rcp2(wl[0]), rir = rcp2(wr[0]);
  const P2<S> g = p2<S>(c.g);
  const P2<S> al = sqrt2((g * wl[4]) * ril);
  const P2<S> ar = sqrt2((g * wr[4]) * rir);
  const P2<S> ul = wl[DIR], ur = wr[DIR];
  const P2<S> sl = min2(ul - al, ur - ar);
  const P2<S> sr = max2(ul + al, ur + ar);
  const P2<S> facl = wl[0] * (sl - ul);
  const P2<S> facr = wr[0] * (sr - ur);
  const P2<S> sm = fma2(neg2(facr), ur, fma2(facl, ul, wr[4] - wl[4])) * rcp2(facl - facr);
  M2 left, star;
  {
    const bool plx = (S)0 <= sl.x, ply = (S)0 <= sl.y;
    const bool prx = !plx && (S)0 >= sr.x, pry = !ply && (S)0 >= sr.y;
    star.x = !plx && !prx;
    star.y = !ply && !pry;
    left.x = plx || (star.x && (S)0 < sm.x);
    left.y = ply || (star.y && (S)0 < sm.y);
    if (!(sl.x == sl.x && sr.x == sr.x && sm.x == sm.x && sl.y == sl.y && sr.y == sr.y && sm.y == sm.y))
      err |= EVORA_ERR_HLLC;
  }
  P2<S> w[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) w[i] = sel2(left, wl[i], wr[i]);
  const P2<S> ri = sel2(left, ril, rir);
  const P2<S> sk = sel2(left, sl, sr);
  const P2<S> fk = sel2(left, facl, facr);
  const P2<S> ud = w[DIR];
  const P2<S> u2 = fma2(w[3], w[3], fma2(w[2], w[2], w[1] * w[1]));
  const P2<S> e = fma2(w[4], p2<S>(c.g1inv), (p2<S>((S)0.5) * w[0]) * u2);   // total energy
  const P2<S> mu = w[0] * ud;                                                // mass flux
  P2<S> ql[5], fl[5];
  ql[0] = w[0];
  ql[1] = w[0] * w[1];
  ql[2] = w[0] * w[2];
  ql[3] = w[0] * w[3];
  ql[4] = e;
  fl[0] = mu;
  fl[1] = mu * w[1];
  fl[2] = mu * w[2];
  fl[3] = mu * w[3];
  fl[DIR] = fl[DIR] + w[4];
  fl[4] = ud * (e + w[4]);
  // star state (statex, riemann.f90:241-288); taken only where `star`
  const P2<S> chi = fk * rcp2(sk - sm);
  P2<S> qx[5];
  qx[0] = chi;
  qx[1] = chi * w[1];
  qx[2] = chi * w[2];
  qx[3] = chi * w[3];
  qx[DIR] = chi * sm;
  qx[4] = chi * fma2(sm - ud, fma2(w[4], rcp2(fk), sm), e * ri);
#pragma unroll
  for (int i = 0; i < 5; ++i) f[i] = sel2(star, fma2(sk, qx[i] - ql[i], fl[i]), fl[i]);
}

// Signal speeds |u_d| + a of two conserved states (the CFL maxima).
template <typename S>
__device__ __forceinline__ void speeds_p(const P2<S>* q, const Gas<S>& c, const HydroParams& P, unsigned& err,
                                         P2<S>* s) {
  P2<S> w[5];
  prim_p(q, w, c, P, err);
  const P2<S> a = sqrt2((p2<S>(c.g) * w[4]) * rcp2(w[0]));
  s[0] = abs2(w[1]) + a;
  s[1] = abs2(w[2]) + a;
  s[2] = abs2(w[3]) + a;
}

}  // namespace evora
