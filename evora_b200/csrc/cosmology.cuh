// cosmology.cuh -- the comoving time integration of the reference and the
// units that follow the expansion factor, as __host__ __device__ functions:
// the host drop-ins (abi.cu) and the single-thread control kernel of a
// resident grid (grid.cu) run the same arithmetic.
//
//   cosmostart          cosmology.f90:26-36
//   compcosmo           cosmology.f90:38-51 (rungekutta 136-163, dcosmodt
//                       111-120, adot2 101-109)
//   cosmostep           timestep.f90:59-70
//   updatetime          timestep.f90:147-171 (both branches)
//   timestepiteration   timestep.f90:173-226
//   comoving units      units.f90:32-63 (temp0, temp0inv, kappa0)
//
// Association is the Fortran one (left to right); a**2.0 is a*a (gcc folds
// pow(a, 2.0) into one correctly rounded product, and so does gfortran).  Every
// user is compiled without FMA contraction (--fmad=false on the device; the
// x86-64 host compiler emits no FMA by default), so the scalars match a
// gfortran build of the reference bit for bit; the one libm power, a**5.0 in
// kappa0, is correctly rounded on the device (pow_rn) and libm's pow on the
// host.
#pragma once

#include <cmath>

#include "hydro_math.cuh"

namespace evora {

// Physical constants of module global (global.f90:98-112).
constexpr double kKb = 1.3806200e-16;
constexpr double kRhoc = 1.88e-29;
constexpr double kAtomicMass = 1.660538782e-24;
constexpr double kMegapc = 3.08568025e24;
constexpr double kKilometer = 1e5;
constexpr int kNdump = EVORA_NDUMP;

// The time scalars (same order as evora_time).
struct CosmoTime {
  double t, dt, cosmo, oldcosmo, cosmodot, expand, redshift;
};

// x^n for a small n >= 1, correctly rounded but for inputs within ~2^-100
// relative of a rounding boundary: the product is carried as a double-double
// (Dekker's exact product through one FMA, then Knuth's fast two-sum; Ogita,
// Rump and Oishi 2005, "Accurate sum and dot product"), so its error before
// the final rounding is a few units of 2^-104.  The FMA here is an explicit
// operation, not a contraction.
__host__ __device__ inline double pow_rn(double x, int n) {
  double h = x, l = 0.0;
  for (int i = 1; i < n; ++i) {
    const double p = h * x;
    double e = std::fma(h, x, -p);   // h x - p, exactly
    e = std::fma(l, x, e);           // + l x
    h = p + e;
    l = e - (h - p);
  }
  return h + l;
}

// adot2(a) = omega0 (1/a - 1) + lambda0 (a^2 - 1) + 1 (cosmology.f90:101-109).
__host__ __device__ inline double adot2(const HydroParams& P, double a) {
  return P.omega0 * (1.0 / a - 1.0) + P.lambda0 * (a * a - 1.0) + 1.0;
}

// dcosmodt(t, a) = a^2 sqrt(adot2(a)) (cosmology.f90:111-120); t unused.
__host__ __device__ inline double dcosmodt(const HydroParams& P, double a) {
  return (a * a) * std::sqrt(adot2(P, a));
}

// rungekutta(f, x, dx, dcosmodt) (cosmology.f90:136-163), as written there:
// the last stage is evaluated at the unadvanced f.
__host__ __device__ inline void rungekutta(const HydroParams& P, double& f, double dx) {
  const double dfdx1 = dcosmodt(P, f);
  const double dx2 = 0.5 * dx;
  double ff = f + dx2 * dfdx1;
  double dfdx2 = dcosmodt(P, ff);
  ff = f + dx2 * dfdx2;
  double dfdx3 = dcosmodt(P, ff);
  dfdx3 = dfdx2 + dfdx3;
  dfdx2 = dcosmodt(P, f);
  f = f + (dfdx1 + dfdx2 + 2.0 * dfdx3) * dx / 6.0;
}

// cosmostart (cosmology.f90:26-36).
__host__ __device__ inline void cosmostart(const HydroParams& P, CosmoTime& s) {
  s.redshift = P.zstart;
  s.cosmo = 1.0 / (1.0 + P.zstart);
  s.cosmodot = dcosmodt(P, s.cosmo);
}

// compcosmo (cosmology.f90:38-51).
__host__ __device__ inline void compcosmo(const HydroParams& P, CosmoTime& s) {
  s.oldcosmo = s.cosmo;
  rungekutta(P, s.cosmo, s.dt);
  s.cosmodot = dcosmodt(P, s.cosmo);
  s.expand = s.cosmo * s.cosmodot;
  s.redshift = 1.0 / s.cosmo - 1.0;
}

// cosmostep (timestep.f90:59-70): dt = min(cosmo / cosmodot c_cosmo, dt).
__host__ __device__ inline void cosmostep(const HydroParams& P, CosmoTime& s, unsigned& err) {
  const double v = s.cosmo / s.cosmodot * P.c_cosmo;
  s.dt = (s.dt < v) ? s.dt : v;
  if (s.dt <= 0.0) err |= EVORA_ERR_DT;
}

// timestepiteration(targetredshift) (timestep.f90:173-226): the step dt
// that brings cosmo from oldcosmo to 1/(1+z), by the reference's regula
// falsi with the Illinois halving, at most 10 rounds.
__host__ __device__ inline void timestepiteration(const HydroParams& P, CosmoTime& s, double z, unsigned& err) {
  const int nit = 10;
  const double tol = 1e-20;
  const double target = 1.0 / (1.0 + z);
  double l = 0.0, r = s.dt;
  double fl = target - s.oldcosmo, fr = target - s.cosmo;
  int side = 0;
  for (int i = 1; i <= nit; ++i) {
    const double m = (fr * l - fl * r) / (fr - fl);
    if (std::fabs(r - l) < tol * std::fabs(r + l)) break;
    s.dt = m;
    s.cosmo = s.oldcosmo;
    compcosmo(P, s);
    const double fm = target - s.cosmo;
    if (std::fabs(fm) < tol) break;
    if (fm * fr > 0.0) {
      r = m;
      fr = fm;
      if (side == -1) fl = fl * 0.5;
      side = -1;
    } else if (fl * fm > 0.0) {
      l = m;
      fl = fm;
      if (side == 1) fr = fr * 0.5;
      side = 1;
    } else {
      break;
    }
    if (i == nit) err |= EVORA_ERR_COSMO;
  }
}

// updatetime(go, dump, k) (timestep.f90:147-171).  dump_redshift holds
// kNdump entries; k is 1-based.
__host__ __device__ inline void updatetime(const HydroParams& P, double tend, const double* dump_redshift,
                                           CosmoTime& s, int& go, int& dump, int k, unsigned& err) {
  if (P.supercomoving) {
    if (s.redshift <= P.zend) {
      timestepiteration(P, s, P.zend, err);
      go = 0;
    } else if (k >= 1 && k <= kNdump && s.redshift < dump_redshift[k - 1]) {
      timestepiteration(P, s, dump_redshift[k - 1], err);
      dump = 1;
    }
  } else if (tend - s.t <= s.dt) {
    s.dt = tend - s.t;
    go = 0;
  }
  s.t = s.t + s.dt;
}

// peeblesint(a) = adot2(a)^(-3/2) (cosmology.f90:122-132).
inline double peeblesint(const HydroParams& P, double a) { return std::pow(adot2(P, a), -1.5); }

// trapezoid(int, a, b, delta, f) (cosmology.f90:165-191): steps of delta
// from a, the last one shortened to end at b.
template <class F>
double trapezoid(double a, double b, double delta, F f) {
  double sum = 0.0, x = a, dx = delta;
  double fr = f(x);
  while (x < b) {
    const double fl = fr;
    if (x + dx > b) {
      dx = b - x;
      x = b;
    } else {
      x = x + dx;
    }
    fr = f(x);
    sum = sum + 0.5 * dx * (fl + fr);
  }
  return sum;
}

// peebles(fpeebles) (cosmology.f90:76-97): the linear growth rate
// d ln D / d ln a at a = cosmo, from the growing mode D ~ adot int da/adot^3.
inline double peebles(const HydroParams& P, double cosmo) {
  const double f1 = (P.lambda0 * (cosmo * cosmo) - 0.5 * P.omega0 / cosmo) / adot2(P, cosmo);
  const double integral = trapezoid(1e-8, cosmo, 1e-8, [&](double a) { return peeblesint(P, a); });
  const double f2 = cosmo * peeblesint(P, cosmo) / integral;
  return f1 + f2 - 1.0;
}

// h, d0, t0, l0, m0 of compunits (units.f90:32-44): the cosmological
// bases with supercomoving (hubble0 * 0.01 with a single-precision 0.01),
// else 1, 1, 1, 1, kb.
inline void unit_bases(const evora_params* p, double b[5]) {
  if (p->supercomoving) {
    const double h = p->hubble0 * (double)0.01f;
    b[0] = h;
    b[1] = p->omega0 * kRhoc * (h * h);
    b[2] = 1.0 / (p->hubble0 * kKilometer / kMegapc);
    b[3] = p->box * kMegapc / h;
    b[4] = kAtomicMass;
  } else {
    b[0] = b[1] = b[2] = b[3] = 1.0;
    b[4] = kKb;
  }
}

// kappa_coef = 4.6d13 * 1d-20 / (37.8 / 40.0) (units.f90:62), the quotient
// in single precision.
inline double kappa_coef() { return 4.6e13 * 1e-20 / (double)(37.8f / 40.0f); }

// compunits (units.f90:32-63), the parts that depend on a with the
// supercomoving branch's h, d0, t0, l0, m0 folded into P.u_*:
//   temp0  = l0^2 / a^2 / t0^2 * m0 / kb
//   kappa0 = a^5 * t0^3 / d0 / l0^4 * 0.5 * kappa_coef
__host__ __device__ inline Units comoving_units(const HydroParams& P, double a) {
  Units u;
  u.temp0 = P.u_l02 / (a * a) / P.u_t02 * P.u_m0 / kKb;
  u.temp0inv = 1.0 / u.temp0;
#ifdef __CUDA_ARCH__
  const double a5 = pow_rn(a, 5);
#else
  const double a5 = std::pow(a, 5.0);
#endif
  u.kappa0 = a5 * P.u_t03 / P.u_d0 / P.u_l04 * 0.5 * P.u_kcoef;
  return u;
}

}  // namespace evora
