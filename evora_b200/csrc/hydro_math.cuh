// hydro_math.cuh -- device arithmetic of the evora hydro update.
//
// Every function states the reference routine it follows.  The association
// of each floating-point expression is the Fortran one (left to right,
// a*b*c = (a*b)*c, x**2 = x*x), so a build without FMA contraction
// (--fmad=false) reproduces a gfortran -O3 x86-64 build of the reference
// bit for bit wherever libm pow is not involved (pow only feeds the entropy
// field S).  Fortran MIN/MAX are "take the next argument if it is
// smaller/larger", written as selects rather than fmin/fmax so that ties of
// signed zeros resolve the same way.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if !defined(__CUDACC__)
// Host compilation of the device arithmetic (used by the CPU emulation of the
// fused kernel in the test suite): the CUDA qualifiers vanish.
#define __host__
#define __device__
#define __forceinline__ inline
#define __global__
#endif

#include "../../include/evora_gpu.h"
#if defined(__CUDACC__) && !defined(EVORA_HOST_EMU)
#include "fast_exp.cuh"
#endif

namespace evora {

// coef(ncool, 2) of module global (rates.f90:26-78): c[i][0] = coef(i+1, 1)
// (chemical), c[i][1] = coef(i+1, 2) (cooling); uv = the background J
// (compbackground, chemistry.f90:123-157).
constexpr int kNcool = 13;
struct ChemCoef {
  double c[kNcool][2];
  double uv;
};

// Step control block of a resident grid, in device memory.  Kernels of a
// step read dt from here and return at once when the step is inactive
// (go was already false, or an error was raised earlier).
struct GridCtl {
  double t, dt, tend;
  int go;        // updatetime's go flag
  int active;    // the current step runs
  long long k;   // steps completed
  unsigned err;  // accumulated EVORA_ERR_* mask
  unsigned errnext;  // errors of the CFL maxima in snext (raised when used)
  unsigned long long smax[3];   // CFL maxima of |u_d| + a (ordered bits)
  unsigned long long snext[3];  // the same, over the state the update wrote
  unsigned long long vcond;     // thermalstep: min over cells of rho / kappa (ordered bits)
  unsigned long long vcool;     // coolstep: min over cells of the cooling time (ordered bits)
  // comoving coordinates: the time scalars of module global (global.f90:86)
  double cosmo, oldcosmo, cosmodot, expand, redshift;
  // the units compunits derives from cosmo (units.f90:46-63), current step
  double temp0, temp0inv, kappa0;
  int dump;      // dump_redshift index whose dump the last step raised (0: none)
  int k4;        // the next dump_redshift index updatetime tests (main.f90:33)
  double dump_redshift[EVORA_NDUMP];
  ChemCoef coef;   // the chemistry's rate coefficients of the current step
};

__device__ __forceinline__ bool ctl_skip(const GridCtl* ctl) {
  return ctl != nullptr && (!ctl->active || ctl->err != 0);
}

// Parameters every kernel reads (module global after compparameter).
struct HydroParams {
  int nx, ny, nz;
  int solver, limiter, boundtype, secondorder, dualenergy;
  int onedimension, twodimension;
  double g, g1, g1inv, gg1, cfl, de_thresh1;
  double dx, dy, dz, dxinv, dyinv, dzinv;
  // thermal conduction (conduction.f90, thermalstep timestep.f90:72-104)
  int conduction, simplekappa;
  double c_cond, kappa0, temp0;
  // pressure floors (chem, chemistry.f90:92-121, plain build)
  int tempfloor, jeansfloor;
  double temp_fl, temp0inv, jeansfloor0;
  // comoving coordinates (cosmology.f90, timestep.f90:59-70, 147-226)
  int supercomoving;
  int expansion;                  // supercomoving and not atomic (main.f90:178)
  double omega0, lambda0, c_cosmo, zstart, zend;
  double g35;                     // 3g - 5 (parameter.f90:231)
  double gravc;                   // grav = 1.5 omega0 (parameter.f90:236-238)
  double fb;
  // a-independent factors of the comoving units (units.f90:32-63): l0^2,
  // t0^2, m0, t0^3, d0, l0^4, kappa_coef and t0
  double u_l02, u_t02, u_m0, u_t03, u_d0, u_l04, u_kcoef, u_t0;
  // chemistry of the CIE build (chemistry.f90, cie.f90, rates.f90)
  int chemistry, cooling, background, bg;
  double j0, c_chem, substep, chiH, chiHe;
  // the cooling time-step limit (coolstep, timestep.f90:106-143)
  int cooldt;
  // the non-equilibrium build's species solver (ncie, ncie.f90:26-149)
  int noncie;
  double c_cooldt;
};

// The units a kernel uses: the grid's current ones when the run is comoving
// (compunits after every compcosmo, main.f90:132-136), else the constants.
struct Units {
  double temp0, temp0inv, kappa0;
};

__host__ __device__ __forceinline__ Units units_of(const HydroParams& P, const GridCtl* ctl) {
  if (P.supercomoving && ctl != nullptr) return Units{ctl->temp0, ctl->temp0inv, ctl->kappa0};
  return Units{P.temp0, P.temp0inv, P.kappa0};
}

template <typename T>
__host__ __device__ __forceinline__ T fmin2(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__host__ __device__ __forceinline__ T fmax2(T a, T b) { return (b > a) ? b : a; }

__device__ __forceinline__ double dpow(double a, double b) { return std::pow(a, b); }
__device__ __forceinline__ float dpow(float a, float b) { return std::pow(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return std::sqrt(a); }
__device__ __forceinline__ float dsqrt(float a) { return std::sqrt(a); }

// The nf (5 or 6) fields of cell i of a SoA state (field stride n) in FP64;
// a sixth field that is not carried reads as 0.  Fully unrolled, so that v
// stays in registers (a loop bounded by the runtime nf would index v
// dynamically and put it in local memory).
template <typename T>
__device__ __forceinline__ void load_cell(const T* __restrict__ q, int64_t n, int nf, int64_t i, double v[6]) {
#pragma unroll
  for (int f = 0; f < 6; ++f) v[f] = (f < nf) ? (double)q[f * n + i] : 0.0;
}

// Gas constants in the working precision.
template <typename T>
struct Gas {
  T g, g1, g1inv, gg1, de_thresh1;
  __host__ __device__ static Gas make(const HydroParams& P) {
    Gas c;
    c.g = (T)P.g; c.g1 = (T)P.g1; c.g1inv = (T)P.g1inv; c.gg1 = (T)P.gg1;
    c.de_thresh1 = (T)P.de_thresh1;
    return c;
  }
};

// pressure(q,press), comp.f90:45-85.  With dualenergy, writes q[4] (S system)
// or q[5] (E system) back.  Raises EVORA_ERR_PRESSURE for p <= 0.
template <typename T>
__device__ __forceinline__ T pressure(T* q, const Gas<T>& c, bool dualenergy, unsigned& err) {
  T m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
  T kin = (T)0.5 * m2 / q[0];
  T press;
  if (dualenergy) {
    T ratio = kin / q[4];
    if (ratio > c.de_thresh1) {
      press = q[5] * dpow(q[0], c.g1);
      q[4] = kin + press * c.g1inv;
    } else {
      press = c.g1 * (q[4] - kin);
      q[5] = press / dpow(q[0], c.g1);
    }
  } else {
    press = c.g1 * (q[4] - kin);
  }
  if (press <= (T)0) err |= EVORA_ERR_PRESSURE;
  return press;
}

// q2w(q,w), comp.f90:26-43.
template <typename T>
__device__ __forceinline__ void q2w(T* q, T* w, const Gas<T>& c, bool dualenergy, unsigned& err) {
  T densinv = (T)1.0 / q[0];
  w[0] = q[0];
  w[1] = q[1] * densinv;
  w[2] = q[2] * densinv;
  w[3] = q[3] * densinv;
  w[4] = pressure(q, c, dualenergy, err);
}

// comp_slope for one field, muscl.f90:115-169.
template <typename T>
__device__ __forceinline__ T slope1(T wl, T w, T wr, int limiter) {
  T dwl = w - wl;
  T dwr = wr - w;
  if (limiter == 1) {                       // minmod, 128-140
    bool lp = dwl >= (T)0, rp = dwr >= (T)0;
    if (lp != rp) return (T)0;
    return rp ? fmin2(dwl, dwr) : fmax2(dwl, dwr);
  } else if (limiter == 2) {                // monotonised central, 141-154
    T dwc = (wr - wl) * (T)0.5;
    bool lp = dwl >= (T)0, rp = dwr >= (T)0;
    if (lp != rp) return (T)0;
    if (rp) return fmin2(fmin2((T)2.0 * dwl, dwc), (T)2.0 * dwr);
    return fmax2(fmax2((T)2.0 * dwl, dwc), (T)2.0 * dwr);
  } else {                                  // van Leer, 155-163
    T pro = dwl * dwr;
    if (pro <= (T)0) return (T)0;
    return (T)2.0 * pro / (dwr + dwl);
  }
}

// The per-direction predictor term a(:,d) of compevo (muscl.f90:100-104 and
// the 1D/2D copies 64-66, 78-84): a = u_d * s; a(5) += g p s(u_d);
// a(u_d) += s(p) / rho.  d = 1..3.
template <typename T>
__device__ __forceinline__ void predictor_term(const T* w, const T* s, int d, T g, T* a) {
#pragma unroll
  for (int f = 0; f < 5; ++f) a[f] = w[d] * s[f];
  a[4] = a[4] + g * w[4] * s[d];
  a[d] = a[d] + s[4] / w[0];
}

// flux(w,f,dir), riemann.f90:157-205.  nf = 5, 6 (the entropy flux) or 12
// (the non-equilibrium build: the species fluxes f(i) = f(1) w(i-1),
// riemann.f90:200-204; w then carries 11 primitives).
template <typename T, int NF>
__device__ __forceinline__ void flux(const T* w, T* f, int dir, const Gas<T>& c) {
  T u2 = w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
  const T ud = w[dir];
  f[0] = w[0] * ud;
  if (dir == 1) {
    f[1] = w[0] * (w[1] * w[1]) + w[4];
    f[2] = w[0] * w[1] * w[2];
    f[3] = w[0] * w[1] * w[3];
  } else if (dir == 2) {
    f[1] = w[0] * w[2] * w[1];
    f[2] = w[0] * (w[2] * w[2]) + w[4];
    f[3] = w[0] * w[2] * w[3];
  } else {
    f[1] = w[0] * w[3] * w[1];
    f[2] = w[0] * w[3] * w[2];
    f[3] = w[0] * (w[3] * w[3]) + w[4];
  }
  f[4] = ud * ((T)0.5 * w[0] * u2 + c.gg1 * w[4]);
  if (NF >= 6) f[5] = ud * w[4] / dpow(w[0], c.g1);
#pragma unroll
  for (int i = 6; i < NF; ++i) f[i] = f[0] * w[i - 1];
}

// state(w,q), riemann.f90:207-239.
template <typename T, int NF>
__device__ __forceinline__ void state(const T* w, T* q, const Gas<T>& c) {
  q[0] = w[0];
  q[1] = w[0] * w[1];
  q[2] = w[0] * w[2];
  q[3] = w[0] * w[3];
  T u2 = (w[1] * w[1]) + (w[2] * w[2]) + (w[3] * w[3]);
  q[4] = (T)0.5 * w[0] * u2 + w[4] / c.g1;
  if (NF >= 6) q[5] = w[4] / dpow(w[0], c.g1);
#pragma unroll
  for (int i = 6; i < NF; ++i) q[i] = w[0] * w[i - 1];   // riemann.f90:233-237
}

// statex(w,qx,s,sm,dir), riemann.f90:241-288.
template <typename T, int NF>
__device__ __forceinline__ void statex(const T* w, T* qx, T s, T sm, int dir, const Gas<T>& c) {
  const T wd = w[dir];
  qx[0] = w[0] * (s - wd) / (s - sm);
  qx[1] = (dir == 1 ? sm : w[1]) * qx[0];
  qx[2] = (dir == 2 ? sm : w[2]) * qx[0];
  qx[3] = (dir == 3 ? sm : w[3]) * qx[0];
  T energy = (T)0.5 * w[0] * ((w[1] * w[1]) + (w[2] * w[2]) + (w[3] * w[3])) + w[4] / c.g1;
  qx[4] = qx[0] * (energy / w[0] + (sm - wd) * (sm + (w[4] / (w[0] * (s - wd)))));
  if (NF >= 6) qx[5] = qx[0] * w[4] / dpow(w[0], c.g);
#pragma unroll
  for (int i = 6; i < NF; ++i) qx[i] = qx[0] * w[i - 1];   // riemann.f90:282-286
}

// hll(wl,wr,f,dir), riemann.f90:47-92.
template <typename T, int NF>
__device__ __forceinline__ void hll(const T* wl, const T* wr, T* f, int dir, const Gas<T>& c,
                                    unsigned& err) {
  if (wl[4] <= (T)0 || wr[4] <= (T)0) err |= EVORA_ERR_RIEMANN_PRESSURE;
  T al = dsqrt(c.g * wl[4] / wl[0]);
  T ar = dsqrt(c.g * wr[4] / wr[0]);
  T sl = fmin2(wl[dir] - al, wr[dir] - ar);
  T sr = fmax2(wl[dir] + al, wr[dir] + ar);
  if ((T)0 < sl) {
    flux<T, NF>(wl, f, dir, c);
  } else if ((T)0 > sr) {
    flux<T, NF>(wr, f, dir, c);
  } else if (sl <= (T)0 && (T)0 <= sr) {
    T fl[NF], fr[NF], ql[NF], qr[NF];
    flux<T, NF>(wl, fl, dir, c);
    flux<T, NF>(wr, fr, dir, c);
    state<T, NF>(wl, ql, c);
    state<T, NF>(wr, qr, c);
#pragma unroll
    for (int i = 0; i < NF; ++i) f[i] = (sr * fl[i] - sl * fr[i] + sl * sr * (qr[i] - ql[i])) / (sr - sl);
  } else {
    err |= EVORA_ERR_HLL;
#pragma unroll
    for (int i = 0; i < NF; ++i) f[i] = (T)0;
  }
}

// hllc(wl,wr,f,dir), riemann.f90:96-153.
template <typename T, int NF>
__device__ __forceinline__ void hllc(const T* wl, const T* wr, T* f, int dir, const Gas<T>& c,
                                     unsigned& err) {
  if (wl[4] <= (T)0 || wr[4] <= (T)0) err |= EVORA_ERR_RIEMANN_PRESSURE;
  T al = dsqrt(c.g * wl[4] / wl[0]);
  T ar = dsqrt(c.g * wr[4] / wr[0]);
  T sl = fmin2(wl[dir] - al, wr[dir] - ar);
  T sr = fmax2(wl[dir] + al, wr[dir] + ar);
  T facl = wl[0] * (sl - wl[dir]);
  T facr = wr[0] * (sr - wr[dir]);
  T sm = (wr[4] - wl[4] + facl * wl[dir] - facr * wr[dir]) / (facl - facr);
  if ((T)0 < sl) {
    flux<T, NF>(wl, f, dir, c);
  } else if ((T)0 > sr) {
    flux<T, NF>(wr, f, dir, c);
  } else {
    // The two star branches share one evaluation: side K with wave speed sk.
    const bool left = (sl < (T)0 && (T)0 < sm);
    const bool right = (sm <= (T)0 && (T)0 < sr);
    if (!(left || right)) {
      err |= EVORA_ERR_HLLC;
#pragma unroll
      for (int i = 0; i < NF; ++i) f[i] = (T)0;
      return;
    }
    const T* wk = left ? wl : wr;
    const T sk = left ? sl : sr;
    T fk[NF], qk[NF], qx[NF];
    flux<T, NF>(wk, fk, dir, c);
    state<T, NF>(wk, qk, c);
    statex<T, NF>(wk, qx, sk, sm, dir, c);
#pragma unroll
    for (int i = 0; i < NF; ++i) f[i] = fk[i] + sk * (qx[i] - qk[i]);
  }
}

// riemannsolver(wl,wr,f,dir), riemann.f90:26-43.
template <typename T, int NF>
__device__ __forceinline__ void riemann(const T* wl, const T* wr, T* f, int dir, int solver,
                                        const Gas<T>& c, unsigned& err) {
  if (solver == 1) hll<T, NF>(wl, wr, f, dir, c, err);
  else hllc<T, NF>(wl, wr, f, dir, c, err);
}

// ------------------------------------------------------------------------
// Fast forms (FP32, and FP64 outside the strict mode).  Same formulas as the
// reference routines above, with the divisions shared through reciprocals
// and the energy flux written as u_d (E + p) from one E; results agree with
// the literal forms to a few ulp per operation (the strict FP64 mode keeps
// the literal forms).

// Reciprocal.  FP32: the fast-math division of its translation unit.  FP64:
// the hardware's approximate reciprocal (rcp.approx.ftz.f64, relative error
// about 1e-6) refined by two Newton steps (the error e becomes e^2, then
// e^4: within an ulp), with no branch: the division's range checks and
// slow-path branch cut the kernels into blocks the scheduler cannot
// interleave.  |x| beyond 2^+-1000 is scaled by 2^-+64 first, and the result
// by the same factor, so that the approximation sees neither a subnormal
// argument nor a subnormal result; 0, inf and NaN give +-inf, +-0 and NaN
// (the refinement's residual is NaN there and the approximation is kept).
__device__ __forceinline__ float rcp_fast(float x) { return 1.0f / x; }
__device__ __forceinline__ double rcp_fast(double x) {
#if defined(__CUDA_ARCH__)
  const double a = fabs(x);
  const double s = a > 0x1p1000 ? 0x1p-64 : (a < 0x1p-1000 ? 0x1p64 : 1.0);
  const double xs = x * s;
  double r0;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r0) : "d"(xs));
  double e = fma(-xs, r0, 1.0);
  double r = fma(r0, e, r0);
  e = fma(-xs, r, 1.0);
  r = fma(r, e, r);
  return (e == e ? r : r0) * s;
#else
  return 1.0 / x;
#endif
}

// Square root.  FP32: the fast-math sqrtf.  FP64: the hardware's approximate
// reciprocal square root (rsqrt.approx.ftz.f64) refined by two Newton steps,
// then sqrt(x) = x y with one correction, x y + y/2 (x - (x y)^2): within an
// ulp, with no branch.  x beyond 2^+-1000 is scaled by 2^-+128 (the result
// by 2^-+64); +-0 and inf return themselves, negative x and NaN give NaN.
__device__ __forceinline__ float sqrt_fast(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_fast(double x) {
#if defined(__CUDA_ARCH__)
  const double si = x > 0x1p1000 ? 0x1p-128 : (x < 0x1p-1000 ? 0x1p128 : 1.0);
  const double so = x > 0x1p1000 ? 0x1p64 : (x < 0x1p-1000 ? 0x1p-64 : 1.0);
  const double xs = x * si;
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(xs));
  double e = fma(-(xs * y), y, 1.0);
  y = fma(0.5 * y, e, y);
  e = fma(-(xs * y), y, 1.0);
  y = fma(0.5 * y, e, y);
  double sq = xs * y;
  const double d = fma(-sq, sq, xs);
  sq = fma(0.5 * y, d, sq);
  return sq == sq ? sq * so : ((xs == 0.0 || xs == HUGE_VAL) ? x : sq);
#else
  return std::sqrt(x);
#endif
}

// Powers for the FP64 fast forms' dual-energy terms, rho^(g-1) and rho^g:
// FP64 x^y = exp(y ln x) with Tang's exponential (fast_exp.cuh; the library's
// logarithm), for x > 0 within a few ulp (|y ln x| 2^-53 from the rounding
// of the product, about 5e-16 for rho in [1e-3, 1e3] and y = 2/3), with no
// branch; x = 0 gives 0 for y > 0, x < 0 NaN.  The library's pow, which
// carries its logarithm in extended precision and branches on special
// cases, made the FP64 dual-energy kernels about 2.5 times slower than the
// plain ones.  FP32: the fast-math powf.
__device__ __forceinline__ float pow_fast(float x, float y) { return std::pow(x, y); }
__device__ __forceinline__ double pow_fast(double x, double y) {
#if defined(__CUDA_ARCH__) && !defined(EVORA_HOST_EMU)
  return exp_global(y * log(x));
#else
  return std::pow(x, y);
#endif
}

// minmod without branches: 0 unless both differences have the same sign,
// else the one of smaller magnitude.
template <typename T>
__device__ __forceinline__ T minmod_fast(T dwl, T dwr) {
  const T m = fmin(fabs(dwl), fabs(dwr));
  return dwl * dwr > (T)0 ? copysign(m, dwl) : (T)0;
}

template <typename T>
__device__ __forceinline__ T slope_fast(T wl, T w, T wr, int limiter) {
  if (limiter == 1) return minmod_fast(w - wl, wr - w);
  return slope1(wl, w, wr, limiter);
}

// q2w with dual energy (comp.f90:26-43, 45-85) in the fast forms: one
// reciprocal of rho, the kin/E switch as kin * (1/E), rho^(g-1) by
// pow_fast; resynchronises E (S system) or S (E system) in q as pressure()
// does.
template <typename T>
__device__ __forceinline__ void q2w_de_fast(T* q, T* w, const Gas<T>& c, unsigned& err) {
  const T densinv = rcp_fast(q[0]);
  w[0] = q[0];
  w[1] = q[1] * densinv;
  w[2] = q[2] * densinv;
  w[3] = q[3] * densinv;
  const T m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
  const T kin = (T)0.5 * m2 * densinv;
  const T pg = pow_fast(q[0], c.g1);
  T press;
  if (kin * rcp_fast(q[4]) > c.de_thresh1) {
    press = q[5] * pg;
    q[4] = kin + press * c.g1inv;
  } else {
    press = c.g1 * (q[4] - kin);
    q[5] = press * rcp_fast(pg);
  }
  if (press <= (T)0) err |= EVORA_ERR_PRESSURE;
  w[4] = press;
}

// q2w with one reciprocal (comp.f90:26-43, 56-71 without dual energy).
template <typename T>
__device__ __forceinline__ void q2w_fast(const T* q, T* w, const Gas<T>& c, unsigned& err) {
  const T densinv = rcp_fast(q[0]);
  w[0] = q[0];
  w[1] = q[1] * densinv;
  w[2] = q[2] * densinv;
  w[3] = q[3] * densinv;
  const T m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
  const T p = c.g1 * (q[4] - (T)0.5 * m2 * densinv);
  if (p <= (T)0) err |= EVORA_ERR_PRESSURE;
  w[4] = p;
}

// predictor term with the 1/rho of the cell given (muscl.f90:100-104).
template <typename T>
__device__ __forceinline__ void predictor_term_fast(const T* w, const T* s, int d, T g, T rinv, T* a) {
#pragma unroll
  for (int f = 0; f < 5; ++f) a[f] = w[d] * s[f];
  a[4] = a[4] + g * w[4] * s[d];
  a[d] = a[d] + s[4] * rinv;
}

// HLLC (riemann.f90:96-153) in the fast form.  DIR = 1..3.
template <typename T, int NF, int DIR>
__device__ __forceinline__ void hllc_fast(const T* wl, const T* wr, T* f, const Gas<T>& c, unsigned& err) {
  if (wl[4] <= (T)0 || wr[4] <= (T)0) err |= EVORA_ERR_RIEMANN_PRESSURE;
  const T ril = rcp_fast(wl[0]), rir = rcp_fast(wr[0]);
  const T al = sqrt_fast(c.g * wl[4] * ril);
  const T ar = sqrt_fast(c.g * wr[4] * rir);
  const T ul = wl[DIR], ur = wr[DIR];
  const T sl = fmin2(ul - al, ur - ar);
  const T sr = fmax2(ul + al, ur + ar);
  const T facl = wl[0] * (sl - ul);
  const T facr = wr[0] * (sr - ur);
  const T sm = (wr[4] - wl[4] + facl * ul - facr * ur) * rcp_fast(facl - facr);
  // the side whose state (or star state) gives the flux.  The reference's
  // branches (riemann.f90:130-150) leave sl == 0 with sm > 0 and sr == 0 with
  // sm <= 0 to its error stop; there the star flux equals the plain left
  // (right) flux, which the fast form takes.  Only NaN speeds remain an error.
  const bool pure_left = (T)0 <= sl;
  const bool pure_right = !pure_left && (T)0 >= sr;
  const bool star = !pure_left && !pure_right;
  const bool left = pure_left || (star && (T)0 < sm);
  if (!(sl == sl && sr == sr && sm == sm)) err |= EVORA_ERR_HLLC;
  const T* w = left ? wl : wr;
  const T ri = left ? ril : rir;
  const T sk = left ? sl : sr;
  const T fk = left ? facl : facr;
  const T ud = w[DIR];
  const T u2 = w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
  const T e = (T)0.5 * w[0] * u2 + w[4] * c.g1inv;   // total energy
  const T mu = w[0] * ud;                            // mass flux
  T fl[6], ql[6];
  ql[0] = w[0];
  ql[1] = w[0] * w[1];
  ql[2] = w[0] * w[2];
  ql[3] = w[0] * w[3];
  ql[4] = e;
  fl[0] = mu;
  fl[1] = mu * w[1];
  fl[2] = mu * w[2];
  fl[3] = mu * w[3];
  fl[DIR] += w[4];
  fl[4] = ud * (e + w[4]);
  T rpg = (T)0;   // 1 / rho^(g-1); 1 / rho^g = rpg / rho
  if (NF == 6) {
    rpg = rcp_fast(pow_fast(w[0], c.g1));
    fl[5] = ud * w[4] * rpg;
    ql[5] = w[4] * rpg;
  }
  if (!star) {
#pragma unroll
    for (int i = 0; i < NF; ++i) f[i] = fl[i];
    return;
  }
  // star state (statex, riemann.f90:241-288)
  const T chi = fk * rcp_fast(sk - sm);           // rho (s - u_d) / (s - sm)
  T qx[6];
  qx[0] = chi;
  qx[1] = chi * w[1];
  qx[2] = chi * w[2];
  qx[3] = chi * w[3];
  qx[DIR] = chi * sm;
  qx[4] = chi * (e * ri + (sm - ud) * (sm + w[4] * rcp_fast(fk)));
  if (NF == 6) qx[5] = chi * w[4] * (rpg * ri);
#pragma unroll
  for (int i = 0; i < NF; ++i) f[i] = fl[i] + sk * (qx[i] - ql[i]);
}

template <typename T, int NF, int DIR>
__device__ __forceinline__ void riemann_fast(const T* wl, const T* wr, T* f, int solver, const Gas<T>& c,
                                             unsigned& err) {
  if (solver == 2) hllc_fast<T, NF, DIR>(wl, wr, f, c, err);
  else hll<T, NF>(wl, wr, f, DIR, c, err);
}

// Interface states of sweep (muscl.f90:199-200, 208-209): the state a cell
// shows on its upper face, w + 0.5 s + evo, and on its lower face,
// w - 0.5 s + evo.
template <typename T>
__device__ __forceinline__ T face_plus(T w, T s, T e) { return w + (T)0.5 * s + e; }
template <typename T>
__device__ __forceinline__ T face_minus(T w, T s, T e) { return w - (T)0.5 * s + e; }

// Positive doubles order like their bit patterns as unsigned integers; the
// CFL reduction keeps maxima of signal speeds that way (atomicMax on u64).
#if defined(__CUDACC__)
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}
#else
inline unsigned long long ordered_bits(double v) {
  unsigned long long u;
  std::memcpy(&u, &v, sizeof u);
  return u;
}
#endif

}  // namespace evora

namespace evora {

// hydrostep, timestep.f90:26-57, part 2: from the per-axis maxima of
// |u_d| + a, v = min(1e6, dx/Sx, dy/Sy, dz/Sz) (equal to the reference's
// running min over cells), dt = min(cfl * v, dt_in); EVORA_ERR_DT if <= 0.
__host__ __device__ inline double cfl_dt(const HydroParams& P, double sx, double sy, double sz,
                                         double dt_in, unsigned& err) {
  double v = 1e6;
  double vx = P.dx / sx, vy = P.dy / sy, vz = P.dz / sz;
  v = fmin2(fmin2(fmin2(vx, vy), vz), v);
  double dt = fmin2(P.cfl * v, dt_in);
  if (dt <= 0.0) err |= EVORA_ERR_DT;
  return dt;
}

// updatetime, timestep.f90:147-171, non-comoving branch.
__host__ __device__ inline void update_time(double tend, double& t, double& dt, int& go) {
  if (tend - t <= dt) {
    dt = tend - t;
    go = 0;
  }
  t = t + dt;
}

}  // namespace evora
