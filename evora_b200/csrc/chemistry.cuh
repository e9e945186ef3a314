// chemistry.cuh -- the chemistry and cooling of the reference's CIE build
// (six primordial species in collisional ionisation equilibrium, with an
// optional UV background), as __host__ __device__ functions for the device
// kernel (chem.cu) and the host-side coefficient set-up:
//
//   compcoef        rates.f90:26-78     rate coefficients from the units
//   comprates       rates.f90:80-158    chemical and cooling rates at T
//   cool            rates.f90:160-189   cooling and heating rates
//   cieabundance    cie.f90:58-85       equilibrium abundances
//   implicitcie     cie.f90:87-112      ... with a UV background
//   rf_cie, fne, cieions  cie.f90:114-217  its electron-density root
//   cie             cie.f90:26-56       abundances and the sub-cycled
//                                       pressure update of the cooling
//   compbackground  chemistry.f90:123-157  the UV background J(z)
//
// The species vector n holds H, H+, He, He+, He++, e- (q(7:12) of the
// reference).  Literals keep the reference's kinds: the default-real ones
// (157809.1, 0.3, -0.6353, 0.35, ...) are single precision, as are mH and
// mHe (global.f90:108-109).  Association is left to right; every user is
// compiled without FMA contraction.
#pragma once

#include <cmath>

#include "cosmology.cuh"
#include "hydro_math.cuh"

namespace evora {

constexpr int kNs = 6, kNchem = 9;
constexpr double kNfloor = 1.0e-40, kRatefloor = 1.0e-40;   // global.f90:125
constexpr double kCieTol = 1e-10;                            // global.f90:127
constexpr int kCieNit = 1000;                                // global.f90:128
constexpr double kMH = (double)1.00794f, kMHe = (double)4.002602f, kGff = 1.5;
// The sub-cycles of one cell's cooling update are bounded here (the
// reference's loop has no bound and does not end when the cooling time is
// 0); reaching the bound raises EVORA_ERR_CHEM.
constexpr int kCoolMaxCycles = 1 << 20;

// The units compcoef reads (units.f90:56-60).
struct ChemUnits {
  double chem0, photo0, cool0, heat0;
};

// chem0, photo0, cool0, heat0 of compunits (units.f90:56-60) at expansion
// factor a from the bases in P (u_*): d0 t0 / a / m0, t0 a^2,
// g1 t0^3 a d0 / l0^2 / m0^2, g1 t0^3 a^4 / l0^2 / m0.
__host__ __device__ inline ChemUnits chem_units(const HydroParams& P, double a) {
  ChemUnits u;
  u.chem0 = P.u_d0 * P.u_t0 / a / P.u_m0;
  u.photo0 = P.u_t0 * (a * a);
#ifdef __CUDA_ARCH__
  const double a4 = pow_rn(a, 4);
#else
  const double a4 = std::pow(a, 4.0);
#endif
  u.cool0 = P.g1 * P.u_t03 * a * P.u_d0 / P.u_l02 / (P.u_m0 * P.u_m0);
  u.heat0 = P.g1 * P.u_t03 * a4 / P.u_l02 / P.u_m0;
  return u;
}

// compcoef (rates.f90:26-78).  Entries the reference never sets stay 0.
__host__ __device__ inline void compcoef(const ChemUnits& u, double uv, ChemCoef& k) {
  for (int i = 0; i < kNcool; ++i) k.c[i][0] = k.c[i][1] = 0.0;
  k.uv = uv;
  k.c[0][0] = u.chem0 * 5.85e-11;
  k.c[0][1] = u.cool0 * 1.27e-21;
  k.c[1][0] = u.chem0 * 2.38e-11;
  k.c[1][1] = u.cool0 * 9.38e-22;
  k.c[2][0] = u.chem0 * 5.68e-12;
  k.c[2][1] = u.cool0 * 4.95e-22;
  k.c[3][0] = u.chem0 * 8.4e-11;
  k.c[3][1] = u.cool0 * 8.7e-27;
  k.c[4][0] = u.chem0 * 1.5e-10;
  k.c[4][1] = u.cool0 * 1.55e-26;
  k.c[5][0] = u.chem0 * 3.36e-10;
  k.c[5][1] = u.cool0 * 3.48e-26;
  k.c[6][0] = u.chem0 * 1.9e-3;
  k.c[6][1] = u.cool0 * 1.24e-13;
  k.c[7][1] = u.cool0 * 7.5e-19;
  k.c[8][1] = u.cool0 * 5.54e-17;
  k.c[9][1] = u.cool0 * 1.42e-27 * kGff;
  k.c[10][0] = u.photo0 * 2.54e8 * uv;
  k.c[10][1] = u.heat0 * 2.54e8 * 7.75e-12 * uv;
  k.c[11][0] = u.photo0 * 2.49e8 * uv;
  k.c[11][1] = u.heat0 * 2.49e8 * 2.19e-11 * uv;
  k.c[12][0] = u.photo0 * 1.60e7 * uv;
  k.c[12][1] = u.heat0 * 1.60e7 * 3.10e-11 * uv;
}

// compbackground (chemistry.f90:123-157): J(z) of background model bg;
// other values of bg leave uv as it was.
__host__ __device__ inline double compbackground(int background, int bg, double j0, double redshift, double cosmo,
                                                 double uv) {
  if (!background) return uv;
  const double z = redshift;
  if (bg == 1) {
    uv = j0;
  } else if (bg == 2) {   // simple model of Black (1981)
    if (z < 6 && z > 3) uv = j0 * 4.0 * cosmo;
    else if (z <= 3 && z > 1) uv = j0;
    else uv = 0.0;
  } else if (bg == 3) {   // after Bianchi et al.
    if (z > 8.0) {
      uv = 1e-5 * j0;
    } else if (z <= 8.0 && z > 6.0) {
      const double reddex = (-z + 6.0) * (double)0.35f;
      uv = 0.5 * j0 * std::pow(10.0, reddex);
    } else if (z <= 6.0 && z > 3.0) {
      const double reddex = (-z + 3.0) * (double)0.1f;
      uv = j0 * std::pow(10.0, reddex);
    } else if (z <= 3.0 && z > 1.0) {
      uv = j0;
    } else if (z <= 1.0) {
      uv = j0 * (double)0.1f * std::pow(10.0, z);
    }
  }
  return uv;
}

// comprates (rates.f90:80-158).  The six powers of T are taken as
// exp(c ln T) from one logarithm (ln(T 1e-3) = ln T + ln 1e-3, ...): the
// sub-cycled cooling evaluates this ~10 times per cell and step, and a power
// costs about a logarithm plus an exponential; the results stay within a
// few ulp of the direct powers.  kRefPow: the reference's own powers
// (pow(T, -1.5), pow(T 1e-3, -0.2), ...), for the post-processor's host
// state vector, whose text output is compared digit for digit.
template <bool kRefPow = false>
__host__ __device__ inline void comprates(double temp, const ChemCoef& k, int background, int cooling,
                                          double* chemrate, double* coolrate) {
  const double lt = kRefPow ? 0.0 : std::log(temp);
  const double temproot = std::sqrt(temp);
  const double tempinv = 1.0 / temp;
  const double temp15 = kRefPow ? std::pow(temp, -1.5) : std::exp(-1.5 * lt);
  const double fec = 1.0 / (1.0 + std::sqrt(temp * 1e-5));
  const double fc1 = temproot * fec;
  const double e1 = std::exp(-((double)157809.1f * tempinv));
  const double e2 = std::exp(-((double)286335.4f * tempinv));
  const double e3 = std::exp(-((double)631515.0f * tempinv));
  const double ln1e3 = -6.907755278982137, ln1e6 = -13.815510557964274;   // ln 1e-3, ln 1e-6
  const double fr = kRefPow ? std::pow(temp * 1e-3, (double)(-0.2f)) / (1.0 + std::pow(temp * 1e-6, (double)0.7f))
                            : std::exp((double)(-0.2f) * (lt + ln1e3)) / (1.0 + std::exp((double)0.7f * (lt + ln1e6)));
  const double fr1 = fr / temproot;
  const double fr2 = fr * temproot;
  const float c3 = 0.3f * (-94000.0f);   // a product of two default reals
  const double edr = std::exp((double)(-470000.0f) * tempinv) * (1.0 + (double)c3 * tempinv);
  const double p6353 = kRefPow ? std::pow(temp, (double)(-0.6353f)) : std::exp((double)(-0.6353f) * lt);
  chemrate[0] = k.c[0][0] * fc1 * e1;
  chemrate[1] = k.c[1][0] * fc1 * e2;
  chemrate[2] = k.c[2][0] * fc1 * e3;
  chemrate[3] = k.c[3][0] * fr1;
  chemrate[4] = k.c[4][0] * p6353 + k.c[6][0] * temp15 * edr;
  chemrate[5] = k.c[5][0] * fr1;
  if (background) {
    chemrate[6] = k.c[10][0];
    chemrate[7] = k.c[11][0];
    chemrate[8] = k.c[12][0];
  } else {
    chemrate[6] = chemrate[7] = chemrate[8] = 0.0;
  }
  if (cooling) {
    const double p3647 = kRefPow ? std::pow(temp, (double)0.3647f) : std::exp((double)0.3647f * lt);
    const double p397 = kRefPow ? std::pow(temp, (double)(-0.397f)) : std::exp((double)(-0.397f) * lt);
    coolrate[0] = k.c[0][1] * fc1 * e1;
    coolrate[1] = k.c[1][1] * fc1 * e2;
    coolrate[2] = k.c[2][1] * fc1 * e3;
    coolrate[3] = k.c[3][1] * fr2;
    coolrate[4] = k.c[4][1] * p3647;
    coolrate[5] = k.c[5][1] * fr2;
    coolrate[6] = k.c[6][1] * temp15 * edr;
    coolrate[7] = k.c[7][1] * fec * std::exp((double)(-118348.0f) * tempinv);
    coolrate[8] = k.c[8][1] * p397 * fec * std::exp((double)(-473638.0f) * tempinv);
    coolrate[9] = k.c[9][1] * temproot;
    if (background) {
      coolrate[10] = k.c[10][1];
      coolrate[11] = k.c[11][1];
      coolrate[12] = k.c[12][1];
    } else {
      coolrate[10] = coolrate[11] = coolrate[12] = 0.0;
    }
  }
}

// cool (rates.f90:160-189): lambda (cooling) and gamma (heating).
__host__ __device__ inline void cool(const double* n, const double* cr, int background, double& lambda,
                                     double& gamma) {
  lambda = cr[0] * n[0] + cr[1] * n[2] + cr[2] * n[3] + cr[3] * n[1] + cr[4] * n[3] + cr[5] * n[4] +
           cr[6] * n[3] + cr[7] * n[0] + cr[8] * n[3] + cr[9] * (n[1] + n[3] + 4.0 * n[4]);
  lambda = lambda * n[5];
  gamma = background ? n[0] * cr[10] + n[2] * cr[11] + n[3] * cr[12] : 0.0;
}

// cieions (cie.f90:194-217).
__host__ __device__ inline void cieions(double nH, double nHe, double ne, const double* cr, double& nHII,
                                        double& nHeII, double& nHeIII) {
  const double ion1 = cr[0] * ne + cr[6];
  const double ion2 = cr[1] * ne + cr[7];
  const double ion3 = cr[2] * ne + cr[8];
  if (ion1 < kRatefloor) {
    nHII = kNfloor;
  } else {
    const double xi1 = cr[3] * ne / ion1;
    nHII = nH / (1.0 + xi1);
  }
  if (ion2 < kRatefloor) {
    nHeII = kNfloor;
    nHeIII = kNfloor;
  } else {
    const double xi2 = cr[4] * ne / ion2;
    if (ion3 < kRatefloor) {
      nHeIII = kNfloor;
      nHeII = nHe / (1.0 + xi2);
    } else {
      const double xi3 = cr[5] * ne / ion3;
      nHeIII = nHe / (1.0 + (xi2 + 1.0) * xi3);
      nHeII = nHe / (1.0 + xi2 + 1.0 / xi3);
    }
  }
}

// fne (cie.f90:181-192): charge balance at electron density ne.
__host__ __device__ inline double fne(double nH, double nHe, double ne, const double* cr) {
  double a, b, c;
  cieions(nH, nHe, ne, cr, a, b, c);
  return a + b + 2 * c - ne;
}

// rf_cie (cie.f90:114-179): regula falsi with the Illinois halving for the
// electron density between in1 and in2.
__host__ __device__ inline double rf_cie(double nH, double nHe, double in1, double in2, const double* cr,
                                         unsigned& err) {
  double l = in1, r = in2;
  double fl = fne(nH, nHe, l, cr), fr = fne(nH, nHe, r, cr);
  double m = 0.0;
  if (fl * fr > 0.0) {
    err |= EVORA_ERR_CHEM;   // no root between in1 and in2
    return m;
  }
  int s = 0;
  for (int i = 1; i <= kCieNit; ++i) {
    m = (fr * l - fl * r) / (fr - fl);
    if (std::fabs(r - l) < kCieTol * std::fabs(r + l)) break;
    const double fm = fne(nH, nHe, m, cr);
    if (fm * fr > 0.0) {
      r = m;
      fr = fm;
      if (s == -1) fl = fl * 0.5;
      s = -1;
    } else if (fl * fm > 0.0) {
      l = m;
      fl = fm;
      if (s == 1) fr = fr * 0.5;
      s = 1;
    } else {
      break;
    }
    if (i == kCieNit) err |= EVORA_ERR_CHEM;   // does not converge
  }
  return m;
}

// ncheck (chemistry.f90:159-176) and n = max(n, nfloor) (cie.f90:81-82).
__host__ __device__ inline void check_floor(double* n, unsigned& err) {
  for (int i = 0; i < kNs - 1; ++i)
    if (!(n[i] >= 0.0 && n[i] <= 1e20)) err |= EVORA_ERR_CHEM;
  for (int i = 0; i < kNs; ++i) n[i] = (kNfloor > n[i]) ? kNfloor : n[i];
}

// cieabundance (cie.f90:58-85), with implicitcie (87-112) under a UV
// background.
__host__ __device__ inline void cieabundance(double nH, double nHe, double* n, const double* cr, int background,
                                             double uv, unsigned& err) {
  if (background && uv > 0.0) {
    const double ne = rf_cie(nH, nHe, kNfloor, nH + 2 * nHe, cr, err);
    double nHII, nHeII, nHeIII;
    cieions(nH, nHe, ne, cr, nHII, nHeII, nHeIII);
    n[0] = nH - nHII;
    n[1] = nHII;
    n[2] = nHe - nHeII - nHeIII;
    n[3] = nHeII;
    n[4] = nHeIII;
    n[5] = ne;
    for (int i = 0; i < kNs; ++i) n[i] = (kNfloor > n[i]) ? kNfloor : n[i];
  } else {
    const double fracH = cr[0] / cr[3];
    const double fracHe1 = cr[1] / cr[4];
    const double fracHe2 = cr[2] / cr[5];
    n[0] = nH / (1.0 + fracH);
    n[1] = n[0] * fracH;
    n[2] = nHe / (1.0 + fracHe1 * (1.0 + fracHe2));
    n[3] = n[2] * fracHe1;
    n[4] = n[3] * fracHe2;
    n[5] = n[1] + n[3] + 2 * n[4];
  }
  check_floor(n, err);
}

// sum(n) in element order (press2temp / temp2press, comp.f90:87-119).
__host__ __device__ inline double nsum(const double* n) { return n[0] + n[1] + n[2] + n[3] + n[4] + n[5]; }

// The parameters of chemistry.f90 a cell update reads.
struct ChemParams {
  int cooling, background;
  double chiH, chiHe;   // rhoH / mH, rhoHe / mHe (initchem, chemistry.f90:36-37)
  double c_chem, substep;
};

// cie (cie.f90:26-56) for one cell: the abundances n at (rho, press) and,
// with cooling, the pressure advanced over dt in sub-cycles of at most
// dt * substep and c_chem times the cooling time.
__host__ __device__ inline void cie(const ChemParams& C, const ChemCoef& k, double temp0, double dt, double rho,
                                    double& press, double* n, unsigned& err) {
  const double nH = C.chiH * rho, nHe = C.chiHe * rho;
  double chemrate[kNchem], coolrate[kNcool];
  if (C.cooling) {
    double ct = 0.0;
    int cycles = 0;
    while (ct < dt) {
      if (++cycles > kCoolMaxCycles) {
        err |= EVORA_ERR_CHEM;
        break;
      }
      const double temp = press / nsum(n) * temp0;
      comprates(temp, k, C.background, 1, chemrate, coolrate);
      cieabundance(nH, nHe, n, chemrate, C.background, k.uv, err);
      double lambda, gamma;
      cool(n, coolrate, C.background, lambda, gamma);
      const double coolio = gamma - lambda;
      const double cooltime = std::fabs(press / coolio);
      double cdt = C.c_chem * cooltime;
      const double rest = dt - ct, cap = dt * C.substep;
      if (rest < cdt) cdt = rest;   // min(c_chem * cooltime, dt - ct, dt * substep)
      if (cap < cdt) cdt = cap;
      ct = ct + cdt;
      press = (press + cdt * gamma) / (1.0 + cdt * lambda / press);
    }
  } else {
    const double temp = press / nsum(n) * temp0;
    comprates(temp, k, C.background, 0, chemrate, coolrate);
    cieabundance(nH, nHe, n, chemrate, C.background, k.uv, err);
  }
}

// coolstep's cell term (timestep.f90:123-130): the cooling time
// |press / (Gamma - Lambda)| at T = press / sum(n) temp0, with n replaced in
// place by the equilibrium abundances at (nH, nHe) -- module global's, the
// last cell's of the last chem or initchem, not this cell's.
__host__ __device__ inline double cool_time(const ChemCoef& k, int background, double temp0, double press,
                                            double nH, double nHe, double* n, unsigned& err) {
  double chemrate[kNchem], coolrate[kNcool];
  const double temp = press / nsum(n) * temp0;
  comprates(temp, k, background, 1, chemrate, coolrate);
  cieabundance(nH, nHe, n, chemrate, background, k.uv, err);
  double lambda, gamma;
  cool(n, coolrate, background, lambda, gamma);
  const double coolio = gamma - lambda;
  return std::fabs(press / coolio);
}

// patankarH (ncie.f90:93-117): the implicit (Patankar) update of n(H),
// n(H+) over cdt at the electron density ne.
__host__ __device__ inline void patankar_h(double* n, double ne, double cdt, const double* r) {
  const double p12 = r[3] * ne * cdt;
  const double p21 = (r[0] * ne + r[6]) * cdt;
  const double d1inv = 1.0 / (1.0 + p21);
  const double d2 = 1.0 + p12;
  const double x2 = (n[1] + p21 * n[0] * d1inv) / (d2 - p21 * p12 * d1inv);
  n[0] = (n[0] + p12 * x2) * d1inv;
  n[1] = x2;
}

// patankarHe (ncie.f90:119-149): the same for n(He), n(He+), n(He++).
__host__ __device__ inline void patankar_he(double* n, double ne, double cdt, const double* r) {
  const double p34 = r[4] * ne * cdt;
  const double p43 = (r[1] * ne + r[7]) * cdt;
  const double p45 = r[5] * ne * cdt;
  const double p54 = (r[2] * ne + r[8]) * cdt;
  const double d3inv = 1.0 / (1.0 + p43);
  const double d4 = 1.0 + p34 + p54;
  const double d5inv = 1.0 / (1.0 + p45);
  const double x4 = (n[1] + p43 * n[0] * d3inv + p45 * n[2] * d5inv) / (d4 - p43 * p34 * d3inv - p45 * p54 * d5inv);
  n[0] = (n[0] + p34 * x4) * d3inv;
  n[2] = (n[2] + p54 * x4) * d5inv;
  n[1] = x4;
}

// ncie (ncie.f90:26-90) for one cell, the non-equilibrium build: sub-cycles
// of cdt = min(dt - ct, c_chem t, dt substep), t the cooling time with
// cooling, else max(n / |dn/dt|) over the five ions and atoms at the first
// cycle's rates (without cooling they are not recomputed); each a Patankar
// update of H and He at the cycle's electron density, then n(e-), ncheck,
// the floor and, with cooling, the pressure update.  Bounded like cie.
__host__ __device__ inline void ncie(const ChemParams& C, const ChemCoef& k, double temp0, double dt,
                                     double& press, double* n, unsigned& err) {
  double chemrate[kNchem], coolrate[kNcool];
  double lambda = 0.0, gamma = 0.0;
  double ct = 0.0;
  int cycles = 0;
  while (ct < dt) {
    if (++cycles > kCoolMaxCycles) {
      err |= EVORA_ERR_CHEM;
      break;
    }
    if (C.cooling || ct == 0.0) comprates(press / nsum(n) * temp0, k, C.background, C.cooling, chemrate, coolrate);
    double tchem;
    if (C.cooling) {
      cool(n, coolrate, C.background, lambda, gamma);
      const double coolio = gamma - lambda;
      tchem = std::fabs(press / coolio);
    } else {
      const double* r = chemrate;
      const double ion1 = (r[0] * n[5] + r[6]) * n[0];
      const double ion2 = (r[1] * n[5] + r[7]) * n[2];
      const double ion3 = (r[2] * n[5] + r[8]) * n[3];
      const double rec1 = r[3] * n[1] * n[5];
      const double rec2 = r[4] * n[3] * n[5];
      const double rec3 = r[5] * n[4] * n[5];
      const double delta[5] = {rec1 - ion1, ion1 - rec1, rec2 - ion2, ion2 - rec2 - ion3 + rec3, ion3 - rec3};
      tchem = -HUGE_VAL;   // maxval: an element is taken when it is larger
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const double x = n[i] / std::fabs(delta[i]);
        if (x > tchem) tchem = x;
      }
    }
    double cdt = dt - ct;   // min(dt - ct, c_chem t, dt substep)
    const double lim = C.c_chem * tchem, cap = dt * C.substep;
    if (lim < cdt) cdt = lim;
    if (cap < cdt) cdt = cap;
    ct = ct + cdt;
    const double ne = n[5];
    patankar_h(n, ne, cdt, chemrate);
    patankar_he(n + 2, ne, cdt, chemrate);
    n[5] = n[1] + n[3] + 2.0 * n[4];
    check_floor(n, err);
    if (C.cooling) press = (press + cdt * gamma) / (1.0 + cdt * lambda / press);
  }
}

// coolstep's limit (timestep.f90:136-141): min(dt, c_cooldt v) from v, the
// smallest cooling time (1e6 when no cell is below it).
__host__ __device__ inline double cool_dt(double c_cooldt, double v, double dt, unsigned& err) {
  const double lim = c_cooldt * v;
  if (lim < dt) dt = lim;
  if (dt <= 0.0) err |= EVORA_ERR_DT;
  return dt;
}

}  // namespace evora
