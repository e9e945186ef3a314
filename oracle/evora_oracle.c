/*
 * evora_oracle.c -- TEST INFRASTRUCTURE ONLY.  Not part of the product.
 *
 * A plain-C, FP64 restatement of the hydro update of evora, used by tests/,
 * by __graft_entry__.smoke() and by the CPU legs of bench.py as the checker
 * and the CPU baseline.  Nothing in evora_b200/ links or calls it.
 *
 * It follows the reference line by line: the same array-of-structures
 * layouts (field index fastest, ghost frames as allocated in main.f90:72-75),
 * the same loop order, and the same association of every floating-point
 * expression (Fortran evaluates a*b*c as (a*b)*c; gfortran -O3 on x86-64
 * emits no FMA, so this file is compiled with -ffp-contract=off).  Integer
 * powers x**2 are written x*x as gfortran expands them; real powers call
 * libm pow.  MIN/MAX are evaluated left to right as "take the next argument
 * if it is smaller (larger)".
 *
 * Pinning: the reference ships no test vectors (its tests only draw plots),
 * and no Fortran compiler exists here, so the reference cannot be run as is.
 * oracle/ref_f2c.py translates the reference's own Fortran sources
 * mechanically into C (oracle/_ref/), and tests/test_oracle_pin.py checks
 * this restatement against that translation bit for bit.
 *
 * The reference stops the program on each error condition; this file
 * records the first error as an EVORA_ERR_* bit and carries on, so that the
 * caller can stop.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/evora_gpu.h"

#define NQ 6
#define NW 5
#define NF 6

/* ------------------------------------------------------ module global -- */
/* The hydro subset of module global (global.f90:44-86), filled by
 * orc_compparameter. */
static struct {
  int nx, ny, nz;
  int solver, limiter, boundtype, secondorder, dualenergy;
  double g, g1, g1inv, gg1, cfl, de_thresh1;
  double dx, dy, dz, dxinv, dyinv, dzinv, x0, y0, z0, volume;
  double tstart, tend;
  int onedimension, twodimension;
  int conduction, simplekappa;
  double c_cond, kappa0, temp0;
  int tempfloor, jeansfloor;
  double temp_fl, temp0inv, jeansfloor0;
  /* comoving coordinates (global.f90:55-57, 86, 137-138) */
  int supercomoving, atomic;
  double c_cosmo, omega0, lambda0, zstart, zend, g35;
  double dump_redshift[EVORA_NDUMP];
  double u_d0, u_t0, u_l0, u_m0;        /* compunits' d0, t0, l0, m0 */
  /* chemistry of the CIE build (global.f90:29-35, 63-67, 131-133): q holds
   * nq = 12 values per cell, q(7:12) the species */
  int nq;
  int chemistry, noncie, cooling, background, bg, cooldt;
  double j0, c_chem, substep, chiH, chiHe, c_cooldt;
  /* module global's nH, nHe: chem and initchem set them per cell
   * (chemistry.f90:50-51, 90-91); coolstep reads them as the last cell of
   * the last such pass left them */
  double nH, nHe;
  double chem0, photo0, cool0, heat0;   /* compunits (units.f90:56-60) */
  double coef[13][2], uv;               /* compcoef (rates.f90), compbackground */
} G;

/* The time scalars of module global (global.f90:86): t, dt, cosmo,
 * oldcosmo, cosmodot, expand, redshift (evora_time's order). */
static struct {
  double t, dt, cosmo, oldcosmo, cosmodot, expand, redshift;
} T;

static const double kKb = 1.3806200e-16;   /* global.f90:103 */

static int orc_err = 0;

static void set_err(int code) {
#pragma omp atomic
  orc_err |= code;
}

int orc_error(void) { return orc_err; }
void orc_clear_error(void) { orc_err = 0; }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Fortran MIN/MAX of two reals, left to right. */
static inline double fmin2(double a, double b) { return (b < a) ? b : a; }
static inline double fmax2(double a, double b) { return (b > a) ? b : a; }

/* ------------------------------------------------------------ cosmology -- */
static inline size_t iq(int i, int j, int k);
static double orc_pressure(double* q);

/* adot2(a), cosmology.f90:101-109 (a**2.0 = a*a, as gcc folds pow(a, 2.0)). */
static double adot2(double a) { return G.omega0 * (1.0 / a - 1.0) + G.lambda0 * (a * a - 1.0) + 1.0; }

/* dcosmodt(t, a), cosmology.f90:111-120 (t is not used). */
static double dcosmodt(double a) { return (a * a) * sqrt(adot2(a)); }

/* rungekutta(f, x, dx, dcosmodt), cosmology.f90:136-163, including its last
 * stage taken at the unadvanced f. */
static void rungekutta(double* f, double dx) {
  const double dfdx1 = dcosmodt(*f);
  const double dx2 = 0.5 * dx;
  double ff = *f + dx2 * dfdx1;
  double dfdx2 = dcosmodt(ff);
  ff = *f + dx2 * dfdx2;
  double dfdx3 = dcosmodt(ff);
  dfdx3 = dfdx2 + dfdx3;
  dfdx2 = dcosmodt(*f);
  *f = *f + (dfdx1 + dfdx2 + 2.0 * dfdx3) * dx / 6;
}

/* peeblesint(a), cosmology.f90:122-132. */
static double peeblesint(double a) { return pow(adot2(a), -1.5); }

/* trapezoid(int, a, b, delta, f), cosmology.f90:165-191. */
static double trapezoid(double a, double b, double delta, double (*f)(double)) {
  double sum = 0.0, x = a, dx = delta, fl, fr = f(x);
  while (x < b) {
    fl = fr;
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

/* peebles(fpeebles), cosmology.f90:76-97, at the time scalars s. */
double orc_peebles(const double* s) {
  const double cosmo = s[2];
  const double f1 = (G.lambda0 * (cosmo * cosmo) - 0.5 * G.omega0 / cosmo) / adot2(cosmo);
  const double integral = trapezoid(1e-8, cosmo, 1e-8, peeblesint);
  const double f2 = cosmo * peeblesint(cosmo) / integral;
  return f1 + f2 - 1.0;
}

/* cosmostart, cosmology.f90:26-36. */
static void orc_cosmostart_(void) {
  T.redshift = G.zstart;
  T.cosmo = 1 / (1 + G.zstart);
  T.cosmodot = dcosmodt(T.cosmo);
}

/* compcosmo, cosmology.f90:38-51. */
static void orc_compcosmo_(void) {
  T.oldcosmo = T.cosmo;
  rungekutta(&T.cosmo, T.dt);
  T.cosmodot = dcosmodt(T.cosmo);
  T.expand = T.cosmo * T.cosmodot;
  T.redshift = 1.0 / T.cosmo - 1.0;
}

/* cosmostep, timestep.f90:59-70. */
static void orc_cosmostep_(void) {
  T.dt = fmin2(T.cosmo / T.cosmodot * G.c_cosmo, T.dt);
  if (T.dt <= 0.0) set_err(EVORA_ERR_DT);
}

/* timestepiteration(targetredshift), timestep.f90:173-226. */
static void orc_timestepiteration_(double targetredshift) {
  const int cosmoend_nit = 10;
  const double cosmoend_tol = 1e-20;
  const double targetcosmo = 1.0 / (1.0 + targetredshift);
  double l = 0.0, r = T.dt;
  double fl = targetcosmo - T.oldcosmo, fr = targetcosmo - T.cosmo;
  int s = 0;
  for (int i = 1; i <= cosmoend_nit; ++i) {
    const double m = (fr * l - fl * r) / (fr - fl);
    if (fabs(r - l) < cosmoend_tol * fabs(r + l)) break;
    T.dt = m;
    T.cosmo = T.oldcosmo;
    orc_compcosmo_();
    const double fm = targetcosmo - T.cosmo;
    if (fabs(fm) < cosmoend_tol) break;
    if (fm * fr > 0.0) {
      r = m; fr = fm;
      if (s == -1) fl = fl * 0.5;
      s = -1;
    } else if (fl * fm > 0.0) {
      l = m; fl = fm;
      if (s == 1) fr = fr * 0.5;
      s = 1;
    } else {
      break;
    }
    if (i == cosmoend_nit) set_err(EVORA_ERR_COSMO);
  }
}

/* compunits, units.f90:46-63: the units the hydro path and the chemistry
 * read (temp0, temp0inv, kappa0, chem0, photo0, cool0, heat0) at the
 * current cosmo. */
static void orc_compunits_(void) {
  const double c = T.cosmo, t0 = G.u_t0, l0 = G.u_l0, d0 = G.u_d0, m0 = G.u_m0;
  G.temp0 = (l0 * l0) / (c * c) / (t0 * t0) * m0 / kKb;
  G.temp0inv = 1.0 / G.temp0;
  const double kappa_coef = 4.6e13 * 1e-20 / (double)(37.8f / 40.0f);
  G.kappa0 = pow(c, 5.0) * pow(t0, 3.0) / d0 / pow(l0, 4.0) * 0.5 * kappa_coef;
  G.chem0 = d0 * t0 / c / m0;
  G.photo0 = t0 * (c * c);
  G.cool0 = G.g1 * pow(t0, 3.0) * c * d0 / (l0 * l0) / (m0 * m0);
  G.heat0 = G.g1 * pow(t0, 3.0) * pow(c, 4.0) / (l0 * l0) / m0;
}

/* ---------------------------------------------------- chemistry (CIE) -- */
/* The CIE build: n = q(7:12) = H, H+, He, He+, He++, e- (global.f90:29-35,
 * 121-133).  Default-real literals are single precision, as in the
 * Fortran. */
static const double kNfloor = 1.0e-40, kRatefloor = 1.0e-40, kCieTol = 1e-10;
static const int kCieNit = 1000;

/* compcoef, rates.f90:26-78 (entries it never sets stay 0). */
static void orc_compcoef_(void) {
  memset(G.coef, 0, sizeof G.coef);
  const double uv = G.uv;
  G.coef[0][0] = G.chem0 * 5.85e-11;   G.coef[0][1] = G.cool0 * 1.27e-21;
  G.coef[1][0] = G.chem0 * 2.38e-11;   G.coef[1][1] = G.cool0 * 9.38e-22;
  G.coef[2][0] = G.chem0 * 5.68e-12;   G.coef[2][1] = G.cool0 * 4.95e-22;
  G.coef[3][0] = G.chem0 * 8.4e-11;    G.coef[3][1] = G.cool0 * 8.7e-27;
  G.coef[4][0] = G.chem0 * 1.5e-10;    G.coef[4][1] = G.cool0 * 1.55e-26;
  G.coef[5][0] = G.chem0 * 3.36e-10;   G.coef[5][1] = G.cool0 * 3.48e-26;
  G.coef[6][0] = G.chem0 * 1.9e-3;     G.coef[6][1] = G.cool0 * 1.24e-13;
  G.coef[7][1] = G.cool0 * 7.5e-19;
  G.coef[8][1] = G.cool0 * 5.54e-17;
  G.coef[9][1] = G.cool0 * 1.42e-27 * 1.5;                 /* gff */
  G.coef[10][0] = G.photo0 * 2.54e8 * uv;  G.coef[10][1] = G.heat0 * 2.54e8 * 7.75e-12 * uv;
  G.coef[11][0] = G.photo0 * 2.49e8 * uv;  G.coef[11][1] = G.heat0 * 2.49e8 * 2.19e-11 * uv;
  G.coef[12][0] = G.photo0 * 1.60e7 * uv;  G.coef[12][1] = G.heat0 * 1.60e7 * 3.10e-11 * uv;
}

/* compbackground, chemistry.f90:123-157. */
static void orc_compbackground_(void) {
  if (!G.background) return;
  const double z = T.redshift, j0 = G.j0;
  if (G.bg == 1) {
    G.uv = j0;
  } else if (G.bg == 2) {
    if (z < 6 && z > 3) G.uv = j0 * 4.0 * T.cosmo;
    else if (z <= 3 && z > 1) G.uv = j0;
    else G.uv = 0.0;
  } else if (G.bg == 3) {
    if (z > 8.0) G.uv = 1e-5 * j0;
    else if (z <= 8.0 && z > 6.0) G.uv = 0.5 * j0 * pow(10.0, (-z + 6.0) * (double)0.35f);
    else if (z <= 6.0 && z > 3.0) G.uv = j0 * pow(10.0, (-z + 3.0) * (double)0.1f);
    else if (z <= 3.0 && z > 1.0) G.uv = j0;
    else if (z <= 1.0) G.uv = j0 * (double)0.1f * pow(10.0, z);
  }
}

/* comprates, rates.f90:80-158: chemical rates r[9], cooling rates cr[13]. */
static void orc_comprates(double temp, double* r, double* cr) {
  const double temproot = sqrt(temp), tempinv = 1.0 / temp, temp15 = pow(temp, -1.5);
  const double fec = 1.0 / (1.0 + sqrt(temp * 1e-5));
  const double fc1 = temproot * fec;
  const double e1 = exp(-((double)157809.1f * tempinv));
  const double e2 = exp(-((double)286335.4f * tempinv));
  const double e3 = exp(-((double)631515.0f * tempinv));
  const double fr = pow(temp * 1e-3, (double)(-0.2f)) / (1.0 + pow(temp * 1e-6, (double)0.7f));
  const double fr1 = fr / temproot, fr2 = fr * temproot;
  const float p3 = 0.3f * (-94000.0f);
  const double edr = exp((double)(-470000.0f) * tempinv) * (1.0 + (double)p3 * tempinv);
  const double (*k)[2] = G.coef;
  r[0] = k[0][0] * fc1 * e1;
  r[1] = k[1][0] * fc1 * e2;
  r[2] = k[2][0] * fc1 * e3;
  r[3] = k[3][0] * fr1;
  r[4] = k[4][0] * pow(temp, (double)(-0.6353f)) + k[6][0] * temp15 * edr;
  r[5] = k[5][0] * fr1;
  r[6] = G.background ? k[10][0] : 0.0;
  r[7] = G.background ? k[11][0] : 0.0;
  r[8] = G.background ? k[12][0] : 0.0;
  if (G.cooling) {
    cr[0] = k[0][1] * fc1 * e1;
    cr[1] = k[1][1] * fc1 * e2;
    cr[2] = k[2][1] * fc1 * e3;
    cr[3] = k[3][1] * fr2;
    cr[4] = k[4][1] * pow(temp, (double)0.3647f);
    cr[5] = k[5][1] * fr2;
    cr[6] = k[6][1] * temp15 * edr;
    cr[7] = k[7][1] * fec * exp((double)(-118348.0f) * tempinv);
    cr[8] = k[8][1] * pow(temp, (double)(-0.397f)) * fec * exp((double)(-473638.0f) * tempinv);
    cr[9] = k[9][1] * temproot;
    cr[10] = G.background ? k[10][1] : 0.0;
    cr[11] = G.background ? k[11][1] : 0.0;
    cr[12] = G.background ? k[12][1] : 0.0;
  }
}

/* cool, rates.f90:160-189. */
static void orc_cool(const double* n, const double* cr, double* lambda, double* gamma) {
  double l = cr[0] * n[0] + cr[1] * n[2] + cr[2] * n[3] + cr[3] * n[1] + cr[4] * n[3] + cr[5] * n[4] +
             cr[6] * n[3] + cr[7] * n[0] + cr[8] * n[3] + cr[9] * (n[1] + n[3] + 4.0 * n[4]);
  *lambda = l * n[5];
  *gamma = G.background ? n[0] * cr[10] + n[2] * cr[11] + n[3] * cr[12] : 0.0;
}

/* cieions, cie.f90:194-217. */
static void orc_cieions(double nH, double nHe, double ne, const double* r, double* nHII, double* nHeII,
                        double* nHeIII) {
  const double ion1 = r[0] * ne + r[6], ion2 = r[1] * ne + r[7], ion3 = r[2] * ne + r[8];
  if (ion1 < kRatefloor) *nHII = kNfloor;
  else *nHII = nH / (1.0 + r[3] * ne / ion1);
  if (ion2 < kRatefloor) {
    *nHeII = kNfloor;
    *nHeIII = kNfloor;
  } else {
    const double xi2 = r[4] * ne / ion2;
    if (ion3 < kRatefloor) {
      *nHeIII = kNfloor;
      *nHeII = nHe / (1.0 + xi2);
    } else {
      const double xi3 = r[5] * ne / ion3;
      *nHeIII = nHe / (1.0 + (xi2 + 1.0) * xi3);
      *nHeII = nHe / (1.0 + xi2 + 1.0 / xi3);
    }
  }
}

/* fne, cie.f90:181-192. */
static double orc_fne(double nH, double nHe, double ne, const double* r) {
  double a, b, c;
  orc_cieions(nH, nHe, ne, r, &a, &b, &c);
  return a + b + 2 * c - ne;
}

/* rf_cie, cie.f90:114-179. */
static double orc_rf_cie(double nH, double nHe, double in1, double in2, const double* r) {
  double l = in1, rr = in2, fl = orc_fne(nH, nHe, l, r), fr = orc_fne(nH, nHe, rr, r), m = 0.0;
  if (fl * fr > 0.0) {
    set_err(EVORA_ERR_CHEM);
    return m;
  }
  int s = 0;
  for (int i = 1; i <= kCieNit; ++i) {
    m = (fr * l - fl * rr) / (fr - fl);
    if (fabs(rr - l) < kCieTol * fabs(rr + l)) break;
    const double fm = orc_fne(nH, nHe, m, r);
    if (fm * fr > 0.0) {
      rr = m; fr = fm;
      if (s == -1) fl = fl * 0.5;
      s = -1;
    } else if (fl * fm > 0.0) {
      l = m; fl = fm;
      if (s == 1) fr = fr * 0.5;
      s = 1;
    } else {
      break;
    }
    if (i == kCieNit) set_err(EVORA_ERR_CHEM);
  }
  return m;
}

/* cieabundance with implicitcie, cie.f90:58-112, and ncheck
 * (chemistry.f90:159-176). */
static void orc_cieabundance(double nH, double nHe, double* n, const double* r) {
  if (G.background && G.uv > 0.0) {
    const double ne = orc_rf_cie(nH, nHe, kNfloor, nH + 2 * nHe, r);
    double a, b, c;
    orc_cieions(nH, nHe, ne, r, &a, &b, &c);
    n[0] = nH - a; n[1] = a; n[2] = nHe - b - c; n[3] = b; n[4] = c; n[5] = ne;
    for (int i = 0; i < 6; ++i) n[i] = fmax2(n[i], kNfloor);
  } else {
    const double fracH = r[0] / r[3], fracHe1 = r[1] / r[4], fracHe2 = r[2] / r[5];
    n[0] = nH / (1.0 + fracH);
    n[1] = n[0] * fracH;
    n[2] = nHe / (1.0 + fracHe1 * (1.0 + fracHe2));
    n[3] = n[2] * fracHe1;
    n[4] = n[3] * fracHe2;
    n[5] = n[1] + n[3] + 2 * n[4];
  }
  for (int i = 0; i < 5; ++i)
    if (!(n[i] >= 0.0 && n[i] <= 1e20)) set_err(EVORA_ERR_CHEM);
  for (int i = 0; i < 6; ++i) n[i] = fmax2(n[i], kNfloor);
}

static double nsum(const double* n) { return n[0] + n[1] + n[2] + n[3] + n[4] + n[5]; }

/* cie(rho, press, n), cie.f90:26-56, over the step T.dt. */
static void orc_cie(double rho, double* press, double* n) {
  const double nH = G.chiH * rho, nHe = G.chiHe * rho;
  double r[9], cr[13];
  if (G.cooling) {
    double ct = 0.0;
    long cycles = 0;
    while (ct < T.dt) {
      if (++cycles > (1L << 20)) {   /* the library's bound (the reference has none) */
        set_err(EVORA_ERR_CHEM);
        break;
      }
      const double temp = *press / nsum(n) * G.temp0;
      orc_comprates(temp, r, cr);
      orc_cieabundance(nH, nHe, n, r);
      double lambda, gamma;
      orc_cool(n, cr, &lambda, &gamma);
      const double coolio = gamma - lambda;
      const double cooltime = fabs(*press / coolio);
      const double cdt = fmin2(fmin2(G.c_chem * cooltime, T.dt - ct), T.dt * G.substep);
      ct = ct + cdt;
      *press = (*press + cdt * gamma) / (1.0 + cdt * lambda / *press);
    }
  } else {
    const double temp = *press / nsum(n) * G.temp0;
    orc_comprates(temp, r, cr);
    orc_cieabundance(nH, nHe, n, r);
  }
}

/* patankarH (ncie.f90:93-117): the implicit (Patankar) update of n(H),
 * n(H+) over cdt at the electron density ne. */
static void orc_patankar_h(double* n, double ne, double cdt, const double* r) {
  const double p12 = r[3] * ne * cdt;
  const double p21 = (r[0] * ne + r[6]) * cdt;
  const double d1inv = 1.0 / (1.0 + p21);
  const double d2 = 1.0 + p12;
  const double x2 = (n[1] + p21 * n[0] * d1inv) / (d2 - p21 * p12 * d1inv);
  const double x1 = (n[0] + p12 * x2) * d1inv;
  n[0] = x1;
  n[1] = x2;
}

/* patankarHe (ncie.f90:119-149): the same for n(He), n(He+), n(He++). */
static void orc_patankar_he(double* n, double ne, double cdt, const double* r) {
  const double p34 = r[4] * ne * cdt;
  const double p43 = (r[1] * ne + r[7]) * cdt;
  const double p45 = r[5] * ne * cdt;
  const double p54 = (r[2] * ne + r[8]) * cdt;
  const double d3inv = 1.0 / (1.0 + p43);
  const double d4 = 1.0 + p34 + p54;
  const double d5inv = 1.0 / (1.0 + p45);
  const double x4 = (n[1] + p43 * n[0] * d3inv + p45 * n[2] * d5inv) / (d4 - p43 * p34 * d3inv - p45 * p54 * d5inv);
  const double x3 = (n[0] + p34 * x4) * d3inv;
  const double x5 = (n[2] + p54 * x4) * d5inv;
  n[0] = x3;
  n[1] = x4;
  n[2] = x5;
}

/* ncie(rho, press, n), ncie.f90:26-90, over the step T.dt: sub-cycles of
 * cdt = min(dt - ct, c_chem t, dt substep), t the cooling time with cooling,
 * else the shortest abundance change time max(n / |dn/dt|) (the rates of
 * the first cycle's T: without cooling they are not recomputed), each a
 * Patankar update of the H and He ions, then the electron density, ncheck,
 * the floor and, with cooling, the pressure update. */
static void orc_ncie(double rho, double* press, double* n) {
  (void)rho;
  double r[9], cr[13], lambda = 0.0, gamma = 0.0;
  double ct = 0.0;
  long cycles = 0;
  while (ct < T.dt) {
    if (++cycles > (1L << 20)) {   /* the library's bound (the reference has none) */
      set_err(EVORA_ERR_CHEM);
      break;
    }
    if (G.cooling || ct == 0.0) orc_comprates(*press / nsum(n) * G.temp0, r, cr);
    double cooltime;
    if (G.cooling) {
      orc_cool(n, cr, &lambda, &gamma);
      const double coolio = gamma - lambda;
      cooltime = fabs(*press / coolio);
    } else {
      const double ion1 = (r[0] * n[5] + r[6]) * n[0];
      const double ion2 = (r[1] * n[5] + r[7]) * n[2];
      const double ion3 = (r[2] * n[5] + r[8]) * n[3];
      const double rec1 = r[3] * n[1] * n[5];
      const double rec2 = r[4] * n[3] * n[5];
      const double rec3 = r[5] * n[4] * n[5];
      const double delta[5] = {rec1 - ion1, ion1 - rec1, rec2 - ion2, ion2 - rec2 - ion3 + rec3, ion3 - rec3};
      cooltime = -HUGE_VAL;   /* maxval, taking an element when it is larger */
      for (int i = 0; i < 5; ++i) {
        const double x = n[i] / fabs(delta[i]);
        if (x > cooltime) cooltime = x;
      }
    }
    const double cdt = fmin2(fmin2(T.dt - ct, G.c_chem * cooltime), T.dt * G.substep);
    ct = ct + cdt;
    const double ne = n[5];
    orc_patankar_h(n, ne, cdt, r);
    orc_patankar_he(n + 2, ne, cdt, r);
    n[5] = n[1] + n[3] + 2.0 * n[4];
    for (int i = 0; i < 5; ++i)   /* ncheck, chemistry.f90:159-176 */
      if (!(n[i] >= 0.0 && n[i] <= 1e20)) set_err(EVORA_ERR_CHEM);
    for (int i = 0; i < 6; ++i) n[i] = fmax2(n[i], kNfloor);
    if (G.cooling) *press = (*press + cdt * gamma) / (1.0 + cdt * lambda / *press);
  }
}

void orc_get_coef(double* out) {
  memcpy(out, G.coef, sizeof G.coef);
  out[26] = G.uv;
}

/* The exported forms: s holds the 7 time scalars (evora_time's order). */
static void get_time(double* s) {
  s[0] = T.t; s[1] = T.dt; s[2] = T.cosmo; s[3] = T.oldcosmo; s[4] = T.cosmodot; s[5] = T.expand;
  s[6] = T.redshift;
}
static void put_time(const double* s) {
  T.t = s[0]; T.dt = s[1]; T.cosmo = s[2]; T.oldcosmo = s[3]; T.cosmodot = s[4]; T.expand = s[5];
  T.redshift = s[6];
}
void orc_get_time(double* s) { get_time(s); }
void orc_cosmostep(double* s) { put_time(s); orc_cosmostep_(); get_time(s); }
void orc_compcosmo(double* s) { put_time(s); orc_compcosmo_(); get_time(s); }

/* updatetime(go,dump,k), timestep.f90:147-171, both branches. */
static void orc_updatetime_(int* go, int* dump, int k) {
  if (G.supercomoving) {
    if (T.redshift <= G.zend) {
      orc_timestepiteration_(G.zend);
      *go = 0;
    } else if (k <= EVORA_NDUMP && T.redshift < G.dump_redshift[k - 1]) {
      orc_timestepiteration_(G.dump_redshift[k - 1]);
      *dump = 1;
    }
  } else if (G.tend - T.t <= T.dt) {
    T.dt = G.tend - T.t;
    *go = 0;
  }
  T.t = T.t + T.dt;
}

void orc_updatetime_cosmo(int* go, int* dump, int k, double* s) {
  put_time(s);
  orc_updatetime_(go, dump, k);
  get_time(s);
}

/* compunits at the scalars s (the units of the step after compcosmo). */
void orc_settime(const double* s) {
  put_time(s);
  orc_compunits_();
  if (G.supercomoving && G.chemistry) {   /* main.f90:134-135 */
    orc_compbackground_();
    orc_compcoef_();
  }
}

void orc_get_units(double* out) {
  out[0] = G.temp0; out[1] = G.temp0inv; out[2] = G.kappa0;
}

/* The time scalars at the start of a run: t = tstart, cosmo = 1
 * (parameter.f90:232-234), cosmostart with supercomoving (main.f90:58), then
 * compunits (main.f90:62). */
static void start_time_(void) {
  memset(&T, 0, sizeof T);
  T.t = G.tstart;
  T.cosmo = 1.0;
  if (G.supercomoving) orc_cosmostart_();
  orc_compunits_();
  G.uv = 0.0;                            /* no compbackground before the loop */
  if (G.chemistry) orc_compcoef_();      /* initchem, chemistry.f90:38 */
}

/* expansion(q), cosmology.f90:53-72, with dt and expand of the time
 * scalars. */
static void orc_expansion_(double* q) {
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double* c = &q[iq(ix, iy, iz)];
        const double press = orc_pressure(c);
        c[4] = c[4] - T.dt * G.g35 * T.expand * press / G.g1;
        c[5] = c[5] - T.dt * G.g35 * T.expand * c[5];
      }
}

void orc_expansion(double* q, const double* s) {
  put_time(s);
  orc_expansion_(q);
}

/* compparameter, parameter.f90:164-265 (hydro subset). */
int orc_compparameter(const evora_params* p) {
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return EVORA_ERR_ARG;
  if (p->nx == 1) return EVORA_ERR_ARG;                 /* x is always swept */
  if (p->nz > 1 && p->ny == 1) return EVORA_ERR_ARG;    /* y ghosts never filled */
  if (p->solver != 1 && p->solver != 2) return EVORA_ERR_SOLVER;
  if (p->limiter < 1 || p->limiter > 3) return EVORA_ERR_LIMITER;
  if (p->boundtype < 1 || p->boundtype > 3) return EVORA_ERR_ARG; /* bound fills nothing else */
  G.nx = p->nx; G.ny = p->ny; G.nz = p->nz;
  G.solver = p->solver; G.limiter = p->limiter; G.boundtype = p->boundtype;
  G.secondorder = p->secondorder != 0; G.dualenergy = p->dualenergy != 0;
  G.g = p->g;
  if (p->atomic) G.g = (double)(5.0f / 3.0f);           /* parameter.f90:169-171 */
  G.cfl = p->cfl;
  G.tstart = p->tstart; G.tend = p->tend;
  /* thermal conduction: only the simplekappa branch of thermalflux is
   * defined without chemistry (conduction.f90:140-144 reads the electron
   * density w2n leaves unset, and a gradient before it is assigned) */
  if (p->conduction && !p->simplekappa) return EVORA_ERR_ARG;
  G.conduction = p->conduction != 0;
  G.simplekappa = p->simplekappa != 0;
  G.c_cond = p->c_cond;
  /* the CIE build (parameter.f90:95-104: no background, cooling or cooling
   * time step without chemistry; initchem: chiH = rhoH / mH with module
   * global's single-precision mH, mHe) */
  if (p->chemistry && p->conduction) return EVORA_ERR_ARG;
  G.chemistry = p->chemistry != 0;
  /* the non-equilibrium build (nf = 12, nw = 11): its chem and initchem
   * only; the hydro routines here advect 6 fields (orc_run refuses it) */
  G.noncie = G.chemistry && p->noncie;
  G.nq = G.chemistry ? 12 : 6;
  G.cooling = G.chemistry && p->cooling;
  G.cooldt = G.cooling && p->cooldt;
  G.c_cooldt = p->c_cooldt;
  G.nH = G.nHe = 0.0;
  G.background = G.chemistry && p->background;
  G.bg = p->bg;
  G.j0 = p->j0; G.c_chem = p->c_chem; G.substep = p->substep;
  G.chiH = p->rhoh / (double)1.00794f;
  G.chiHe = p->rhohe / (double)4.002602f;
  G.supercomoving = p->supercomoving != 0;
  G.atomic = p->atomic != 0;
  G.c_cosmo = p->c_cosmo; G.omega0 = p->omega0; G.lambda0 = p->lambda0;
  G.zstart = p->zstart; G.zend = p->zend;
  memcpy(G.dump_redshift, p->dump_redshift, sizeof G.dump_redshift);
  if (G.supercomoving) {
    /* compunits' bases, units.f90:32-38 (0.01 is single precision) */
    const double rhoc = 1.88e-29, megapc = 3.08568025e24, kilometer = 1e5, atomicmass = 1.660538782e-24;
    const double h = p->hubble0 * (double)0.01f;
    G.u_d0 = p->omega0 * rhoc * pow(h, 2.0);
    G.u_t0 = 1.0 / (p->hubble0 * kilometer / megapc);
    G.u_l0 = p->box * megapc / h;
    G.u_m0 = atomicmass;
  } else {
    /* units.f90:39-44: h = d0 = t0 = l0 = 1, m0 = kb */
    G.u_d0 = 1.0; G.u_t0 = 1.0; G.u_l0 = 1.0; G.u_m0 = kKb;
  }
  G.tempfloor = p->tempfloor != 0;
  G.jeansfloor = p->jeansfloor != 0;
  G.temp_fl = p->temp_fl;
  G.onedimension = (p->ny == 1 && p->nz == 1);          /* parameter.f90:173-177 */
  G.twodimension = (p->nz == 1);                        /* parameter.f90:178-182 */
  double xmin = p->xmin, xmax = p->xmax, ymin = p->ymin, ymax = p->ymax;
  double zmin = p->zmin, zmax = p->zmax;
  G.dx = (xmax - xmin) / p->nx;                         /* parameter.f90:192-194 */
  G.dy = (ymax - ymin) / p->ny;
  G.dz = (zmax - zmin) / p->nz;
  if (G.onedimension) {                                 /* parameter.f90:195-205 */
    G.dy = G.dx; G.dz = G.dx;
    ymin = 0.0; ymax = G.dy; zmin = 0.0; zmax = G.dz;
    G.dy = (ymax - ymin) / p->ny;
    G.dz = (zmax - zmin) / p->nz;
  }
  if (G.twodimension) {                                 /* parameter.f90:206-212 */
    G.dz = G.dx;
    zmin = 0.0; zmax = G.dz;
    G.dz = (zmax - zmin) / p->nz;
  }
  G.dxinv = 1.0 / G.dx; G.dyinv = 1.0 / G.dy; G.dzinv = 1.0 / G.dz;
  G.x0 = xmin + G.dx / 2; G.y0 = ymin + G.dy / 2; G.z0 = zmin + G.dz / 2;
  G.volume = (xmax - xmin) * (ymax - ymin) * (zmax - zmin);
  G.g1 = G.g - 1.0;                                     /* parameter.f90:227-231 */
  G.g1inv = 1.0 / G.g1;
  G.gg1 = G.g / G.g1;
  G.de_thresh1 = G.dualenergy ? 1.0 - p->de_thresh : 1.0; /* parameter.f90:244-248 */
  {
    /* compunits after compparameter (main.f90:52-62): jeans0 = sqrt(pi g fb)
     * with module global's single-precision pi and the gas constant g, and
     * the Jeans floor (dx / jeans0 / c_jeans)^2 (units.f90:66-71) */
    const double jeans0 = sqrt((double)3.1415927f * G.g * p->fb);
    G.jeansfloor0 = p->jeansfloor ? (G.dx / jeans0 / p->c_jeans) * (G.dx / jeans0 / p->c_jeans) : 0.0;
  }
  G.g35 = 3.0 * G.g - 5.0;                              /* parameter.f90:231 */
  start_time_();
  return 0;
}

void orc_get_derived(evora_derived* d) {
  d->g = G.g; d->g1 = G.g1; d->g1inv = G.g1inv; d->gg1 = G.gg1; d->cfl = G.cfl;
  d->de_thresh1 = G.de_thresh1;
  d->dx = G.dx; d->dy = G.dy; d->dz = G.dz;
  d->dxinv = G.dxinv; d->dyinv = G.dyinv; d->dzinv = G.dzinv;
  d->x0 = G.x0; d->y0 = G.y0; d->z0 = G.z0; d->volume = G.volume;
  d->onedimension = G.onedimension; d->twodimension = G.twodimension;
}

/* --------------------------------------------------------- array index -- */
/* q(nq, 1:nx, 1:ny, 1:nz) */
static inline size_t iq(int i, int j, int k) {
  return (size_t)G.nq * ((size_t)(i - 1) + (size_t)G.nx * ((size_t)(j - 1) + (size_t)G.ny * (size_t)(k - 1)));
}
/* w(nw, -1:nx+2, -1:ny+2, -1:nz+2) */
static inline size_t iw(int i, int j, int k) {
  return (size_t)NW * ((size_t)(i + 1) + (size_t)(G.nx + 4) * ((size_t)(j + 1) + (size_t)(G.ny + 4) * (size_t)(k + 1)));
}
/* evo(nw, 0:nx+1, 0:ny+1, 0:nz+1) */
static inline size_t ie(int i, int j, int k) {
  return (size_t)NW * ((size_t)i + (size_t)(G.nx + 2) * ((size_t)j + (size_t)(G.ny + 2) * (size_t)k));
}
/* s(nw, 3, 0:nx+1, 0:ny+1, 0:nz+1); d = 1..3 */
static inline size_t is_(int d, int i, int j, int k) {
  return (size_t)NW * ((size_t)(d - 1) + 3 * ((size_t)i + (size_t)(G.nx + 2) * ((size_t)j + (size_t)(G.ny + 2) * (size_t)k)));
}

void orc_array_sizes(int64_t* nq, int64_t* nw, int64_t* ne, int64_t* ns) {
  *nq = (int64_t)G.nq * G.nx * G.ny * G.nz;
  *nw = (int64_t)NW * (G.nx + 4) * (G.ny + 4) * (G.nz + 4);
  *ne = (int64_t)NW * (G.nx + 2) * (G.ny + 2) * (G.nz + 2);
  *ns = (int64_t)NW * 3 * (G.nx + 2) * (G.ny + 2) * (G.nz + 2);
}

/* ------------------------------------------------------------ comp.f90 -- */
/* pressure(q,press), comp.f90:45-85 (may write q(5) or q(6)). */
static double orc_pressure(double* q) {
  double m2 = (q[1] * q[1]) + (q[2] * q[2]) + (q[3] * q[3]);
  double kin = 0.5 * m2 / q[0];
  double ratio = kin / q[4];
  double press;
  if (G.dualenergy) {
    if (ratio > G.de_thresh1) {            /* S - system */
      press = q[5] * pow(q[0], G.g1);
      q[4] = kin + press * G.g1inv;
    } else {                               /* E - system */
      press = G.g1 * (q[4] - kin);
      q[5] = press / pow(q[0], G.g1);
    }
  } else {
    press = G.g1 * (q[4] - kin);
  }
  if (press <= 0.0) set_err(EVORA_ERR_PRESSURE);
  return press;
}

/* q2w(q,w), comp.f90:26-43 (nw = 5: no species loop). */
static void orc_q2w(double* q, double* w) {
  double densinv = 1.0 / q[0];
  w[0] = q[0];
  w[1] = q[1] * densinv;
  w[2] = q[2] * densinv;
  w[3] = q[3] * densinv;
  w[4] = orc_pressure(q);
}

/* ----------------------------------------------------------- muscl.f90 -- */
/* primitive(w,q), muscl.f90:26-43. */
void orc_primitive(double* w, double* q) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
#pragma omp parallel for schedule(static) if (nz > 1)
  for (int iz = 1; iz <= nz; ++iz)
    for (int iy = 1; iy <= ny; ++iy)
      for (int ix = 1; ix <= nx; ++ix) orc_q2w(&q[iq(ix, iy, iz)], &w[iw(ix, iy, iz)]);
}

/* bound(w), boundary.f90:26-113.  Copy of a full ghost-inclusive plane;
 * sign = -1 negates the three velocity components (reflection). */
static void copy_xplane(double* w, int dst, int src, int reflect) {
  for (int k = -1; k <= G.nz + 2; ++k)
    for (int j = -1; j <= G.ny + 2; ++j) {
      double* d = &w[iw(dst, j, k)];
      const double* s = &w[iw(src, j, k)];
      d[0] = s[0];
      d[1] = reflect ? -s[1] : s[1];
      d[2] = reflect ? -s[2] : s[2];
      d[3] = reflect ? -s[3] : s[3];
      d[4] = s[4];
    }
}
static void copy_yplane(double* w, int dst, int src) {
  for (int k = -1; k <= G.nz + 2; ++k)
    for (int i = -1; i <= G.nx + 2; ++i)
      memcpy(&w[iw(i, dst, k)], &w[iw(i, src, k)], NW * sizeof(double));
}
static void copy_zplane(double* w, int dst, int src) {
  for (int j = -1; j <= G.ny + 2; ++j)
    for (int i = -1; i <= G.nx + 2; ++i)
      memcpy(&w[iw(i, j, dst)], &w[iw(i, j, src)], NW * sizeof(double));
}

void orc_bound(double* w) {
  const int nx = G.nx, ny = G.ny, nz = G.nz, bt = G.boundtype;
  /* index bounds of a single rank: lx=1, mx=nx, lx0=2, mx0=nx-1,
   * lx1=0, lx2=-1, mx1=nx+1, mx2=nx+2 (parallel.f90:26-66) */
  if (nx != 1) {                                      /* boundary.f90:33-66 */
    if (bt == 1 || bt == 3) {          /* lower: zero gradient (the reflecting
                                          branch at 41-48 is unreachable) */
      copy_xplane(w, -1, 2, 0);
      copy_xplane(w, 0, 1, 0);
    } else if (bt == 2) {
      copy_xplane(w, -1, nx - 1, 0);
      copy_xplane(w, 0, nx, 0);
    }
    if (bt == 1) {
      copy_xplane(w, nx + 2, nx - 1, 0);
      copy_xplane(w, nx + 1, nx, 0);
    } else if (bt == 2) {
      copy_xplane(w, nx + 2, 2, 0);
      copy_xplane(w, nx + 1, 1, 0);
    } else if (bt == 3) {              /* reflecting upper x face */
      copy_xplane(w, nx + 1, nx, 1);
      copy_xplane(w, nx + 2, nx - 1, 1);
    }
  }
  if (ny != 1) {                                      /* boundary.f90:69-88 */
    if (bt == 1 || bt == 3) {
      copy_yplane(w, -1, 2);
      copy_yplane(w, 0, 1);
      copy_yplane(w, ny + 2, ny - 1);
      copy_yplane(w, ny + 1, ny);
    } else if (bt == 2) {
      copy_yplane(w, -1, ny - 1);
      copy_yplane(w, 0, ny);
      copy_yplane(w, ny + 2, 2);
      copy_yplane(w, ny + 1, 1);
    }
  }
  if (nz != 1) {                                      /* boundary.f90:91-111 */
    if (bt == 1 || bt == 3) {
      copy_zplane(w, -1, 2);
      copy_zplane(w, 0, 1);
      copy_zplane(w, nz + 2, nz - 1);
      copy_zplane(w, nz + 1, nz);
    } else if (bt == 2) {              /* mpisize == 1 */
      copy_zplane(w, -1, nz - 1);
      copy_zplane(w, 0, nz);
      copy_zplane(w, nz + 2, 2);
      copy_zplane(w, nz + 1, 1);
    }
  }
}

/* comp_slope(wl,w,wr,s), muscl.f90:115-169. */
static void orc_comp_slope(const double* wl, const double* w, const double* wr, double* s) {
  double dwl[NW], dwr[NW];
  for (int i = 0; i < NW; ++i) {
    dwl[i] = w[i] - wl[i];
    dwr[i] = wr[i] - w[i];
  }
  if (G.limiter == 1) {                               /* minmod */
    for (int i = 0; i < NW; ++i) {
      int lp = dwl[i] >= 0.0, rp = dwr[i] >= 0.0;
      if (lp != rp) s[i] = 0.0;
      else if (rp) s[i] = fmin2(dwl[i], dwr[i]);
      else s[i] = fmax2(dwl[i], dwr[i]);
    }
  } else if (G.limiter == 2) {                        /* moncen */
    for (int i = 0; i < NW; ++i) {
      double dwc = (wr[i] - wl[i]) * 0.5;
      int lp = dwl[i] >= 0.0, rp = dwr[i] >= 0.0;
      if (lp != rp) s[i] = 0.0;
      else if (rp) s[i] = fmin2(fmin2(2.0 * dwl[i], dwc), 2.0 * dwr[i]);
      else s[i] = fmax2(fmax2(2.0 * dwl[i], dwc), 2.0 * dwr[i]);
    }
  } else if (G.limiter == 3) {                        /* van Leer */
    for (int i = 0; i < NW; ++i) {
      double pro = dwl[i] * dwr[i];
      if (pro <= 0.0) s[i] = 0.0;
      else s[i] = 2.0 * pro / (dwr[i] + dwl[i]);
    }
  } else {
    set_err(EVORA_ERR_LIMITER);
  }
}

/* compevo(w,evo,s), muscl.f90:45-113. */
void orc_compevo(const double* w, double* evo, double* s, double dt) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const double dt2 = -0.5 * dt;
  const double g = G.g;
  if (G.onedimension) {                               /* muscl.f90:60-69 */
    for (int ix = 0; ix <= nx + 1; ++ix) {
      double* sx = &s[is_(1, ix, 1, 1)];
      const double* wc = &w[iw(ix, 1, 1)];
      double a[NW];
      orc_comp_slope(&w[iw(ix - 1, 1, 1)], wc, &w[iw(ix + 1, 1, 1)], sx);
      for (int f = 0; f < NW; ++f) a[f] = wc[1] * sx[f];
      a[4] = a[4] + g * wc[4] * sx[1];
      a[1] = a[1] + sx[4] / wc[0];
      double* e = &evo[ie(ix, 1, 1)];
      for (int f = 0; f < NW; ++f) e[f] = dt2 * a[f] * G.dxinv;
    }
  } else if (G.twodimension) {                        /* muscl.f90:70-88 */
    for (int iy = 0; iy <= ny + 1; ++iy)
      for (int ix = 0; ix <= nx + 1; ++ix) {
        double* s1 = &s[is_(1, ix, iy, 1)];
        double* s2 = &s[is_(2, ix, iy, 1)];
        const double* wc = &w[iw(ix, iy, 1)];
        double a1[NW], a2[NW];
        orc_comp_slope(&w[iw(ix - 1, iy, 1)], wc, &w[iw(ix + 1, iy, 1)], s1);
        orc_comp_slope(&w[iw(ix, iy - 1, 1)], wc, &w[iw(ix, iy + 1, 1)], s2);
        for (int f = 0; f < NW; ++f) a1[f] = wc[1] * s1[f];
        a1[4] = a1[4] + g * wc[4] * s1[1];
        a1[1] = a1[1] + s1[4] / wc[0];
        for (int f = 0; f < NW; ++f) a2[f] = wc[2] * s2[f];
        a2[4] = a2[4] + g * wc[4] * s2[2];
        a2[2] = a2[2] + s2[4] / wc[0];
        double* e = &evo[ie(ix, iy, 1)];
        for (int f = 0; f < NW; ++f) e[f] = dt2 * (a1[f] * G.dxinv + a2[f] * G.dyinv);
      }
  } else {                                            /* muscl.f90:89-111 */
#pragma omp parallel for schedule(static)
    for (int iz = 0; iz <= nz + 1; ++iz)
      for (int iy = 0; iy <= ny + 1; ++iy)
        for (int ix = 0; ix <= nx + 1; ++ix) {
          const double* wc = &w[iw(ix, iy, iz)];
          double* sd[3] = {&s[is_(1, ix, iy, iz)], &s[is_(2, ix, iy, iz)], &s[is_(3, ix, iy, iz)]};
          double a[3][NW];
          orc_comp_slope(&w[iw(ix - 1, iy, iz)], wc, &w[iw(ix + 1, iy, iz)], sd[0]);
          orc_comp_slope(&w[iw(ix, iy - 1, iz)], wc, &w[iw(ix, iy + 1, iz)], sd[1]);
          orc_comp_slope(&w[iw(ix, iy, iz - 1)], wc, &w[iw(ix, iy, iz + 1)], sd[2]);
          for (int i = 0; i < 3; ++i) {
            for (int f = 0; f < NW; ++f) a[i][f] = wc[i + 1] * sd[i][f];
            a[i][4] = a[i][4] + g * wc[4] * sd[i][i + 1];
            a[i][i + 1] = a[i][i + 1] + sd[i][4] / wc[0];
          }
          double* e = &evo[ie(ix, iy, iz)];
          for (int f = 0; f < NW; ++f)
            e[f] = dt2 * (a[0][f] * G.dxinv + a[1][f] * G.dyinv + a[2][f] * G.dzinv);
        }
  }
}

/* --------------------------------------------------------- riemann.f90 -- */
/* flux(w,f,dir), riemann.f90:157-205. */
static void orc_flux(const double* w, double* f, int dir) {
  double u2 = w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
  if (dir == 1) {
    f[0] = w[0] * w[1];
    f[1] = w[0] * (w[1] * w[1]) + w[4];
    f[2] = w[0] * w[1] * w[2];
    f[3] = w[0] * w[1] * w[3];
    f[4] = w[1] * (0.5 * w[0] * u2 + G.gg1 * w[4]);
    f[5] = w[1] * w[4] / pow(w[0], G.g1);
  } else if (dir == 2) {
    f[0] = w[0] * w[2];
    f[1] = w[0] * w[2] * w[1];
    f[2] = w[0] * (w[2] * w[2]) + w[4];
    f[3] = w[0] * w[2] * w[3];
    f[4] = w[2] * (0.5 * w[0] * u2 + G.gg1 * w[4]);
    f[5] = w[2] * w[4] / pow(w[0], G.g1);
  } else {
    f[0] = w[0] * w[3];
    f[1] = w[0] * w[3] * w[1];
    f[2] = w[0] * w[3] * w[2];
    f[3] = w[0] * (w[3] * w[3]) + w[4];
    f[4] = w[3] * (0.5 * w[0] * u2 + G.gg1 * w[4]);
    f[5] = w[3] * w[4] / pow(w[0], G.g1);
  }
}

/* state(w,q), riemann.f90:207-239. */
static void orc_state(const double* w, double* q) {
  q[0] = w[0];
  q[1] = w[0] * w[1];
  q[2] = w[0] * w[2];
  q[3] = w[0] * w[3];
  double u2 = (w[1] * w[1]) + (w[2] * w[2]) + (w[3] * w[3]);
  q[4] = 0.5 * w[0] * u2 + w[4] / G.g1;
  q[5] = w[4] / pow(w[0], G.g1);
}

/* statex(w,qx,s,sm,dir), riemann.f90:241-288. */
static void orc_statex(const double* w, double* qx, double s, double sm, int dir) {
  const double wd = w[dir];
  qx[0] = w[0] * (s - wd) / (s - sm);
  if (dir == 1) {
    qx[1] = sm * qx[0];
    qx[2] = w[2] * qx[0];
    qx[3] = w[3] * qx[0];
  } else if (dir == 2) {
    qx[1] = w[1] * qx[0];
    qx[2] = sm * qx[0];
    qx[3] = w[3] * qx[0];
  } else {
    qx[1] = w[1] * qx[0];
    qx[2] = w[2] * qx[0];
    qx[3] = sm * qx[0];
  }
  double energy = 0.5 * w[0] * ((w[1] * w[1]) + (w[2] * w[2]) + (w[3] * w[3])) + w[4] / G.g1;
  qx[4] = qx[0] * (energy / w[0] + (sm - wd) * (sm + (w[4] / (w[0] * (s - wd)))));
  qx[5] = qx[0] * w[4] / pow(w[0], G.g);
}

/* hll(wl,wr,f,dir), riemann.f90:47-92. */
static void orc_hll(const double* wl, const double* wr, double* f, int dir) {
  if (wl[4] <= 0 || wr[4] <= 0) set_err(EVORA_ERR_RIEMANN_PRESSURE);
  double al = sqrt(G.g * wl[4] / wl[0]);
  double ar = sqrt(G.g * wr[4] / wr[0]);
  double sl = fmin2(wl[dir] - al, wr[dir] - ar);
  double sr = fmax2(wl[dir] + al, wr[dir] + ar);
  if (0 < sl) {
    orc_flux(wl, f, dir);
  } else if (0 > sr) {
    orc_flux(wr, f, dir);
  } else if (sl <= 0 && 0 <= sr) {
    double fl[NF], fr[NF], ql[NQ], qr[NQ];
    orc_flux(wl, fl, dir);
    orc_flux(wr, fr, dir);
    orc_state(wl, ql);
    orc_state(wr, qr);
    for (int i = 0; i < NF; ++i)
      f[i] = (sr * fl[i] - sl * fr[i] + sl * sr * (qr[i] - ql[i])) / (sr - sl);
  } else {
    set_err(EVORA_ERR_HLL);
    for (int i = 0; i < NF; ++i) f[i] = 0.0;
  }
}

/* hllc(wl,wr,f,dir), riemann.f90:96-153. */
static void orc_hllc(const double* wl, const double* wr, double* f, int dir) {
  if (wl[4] <= 0 || wr[4] <= 0) set_err(EVORA_ERR_RIEMANN_PRESSURE);
  double al = sqrt(G.g * wl[4] / wl[0]);
  double ar = sqrt(G.g * wr[4] / wr[0]);
  double sl = fmin2(wl[dir] - al, wr[dir] - ar);
  double sr = fmax2(wl[dir] + al, wr[dir] + ar);
  double facl = wl[0] * (sl - wl[dir]);
  double facr = wr[0] * (sr - wr[dir]);
  double sm = (wr[4] - wl[4] + facl * wl[dir] - facr * wr[dir]) / (facl - facr);
  if (0 < sl) {
    orc_flux(wl, f, dir);
  } else if (0 > sr) {
    orc_flux(wr, f, dir);
  } else if (sl < 0 && 0 < sm) {
    double fl[NF], ql[NQ], qx[NQ];
    orc_flux(wl, fl, dir);
    orc_state(wl, ql);
    orc_statex(wl, qx, sl, sm, dir);
    for (int i = 0; i < NF; ++i) f[i] = fl[i] + sl * (qx[i] - ql[i]);
  } else if (sm <= 0 && 0 < sr) {
    double fr[NF], qr[NQ], qx[NQ];
    orc_flux(wr, fr, dir);
    orc_state(wr, qr);
    orc_statex(wr, qx, sr, sm, dir);
    for (int i = 0; i < NF; ++i) f[i] = fr[i] + sr * (qx[i] - qr[i]);
  } else {
    set_err(EVORA_ERR_HLLC);
    for (int i = 0; i < NF; ++i) f[i] = 0.0;
  }
}

/* riemannsolver(wl,wr,f,dir), riemann.f90:26-43. */
static void orc_riemann(const double* wl, const double* wr, double* f, int dir) {
  if (G.solver == 1) orc_hll(wl, wr, f, dir);
  else if (G.solver == 2) orc_hllc(wl, wr, f, dir);
  else set_err(EVORA_ERR_SOLVER);
}

/* Single interface flux for tests: wl, wr are primitive 5-vectors. */
void orc_riemann_single(const double* wl, const double* wr, double* f, int dir) {
  orc_riemann(wl, wr, f, dir);
}

/* integration(fl,fr,q,delta), muscl.f90:276-290 (nf = 6). */
static inline void orc_integration(const double* fl, const double* fr, double* q, double delta) {
  for (int i = 0; i < NF; ++i) q[i] = q[i] + delta * (fl[i] - fr[i]);
}

/* Left face state of the interface (a|b) along axis d: w + 0.5 s + evo. */
static inline void face_left(const double* w, const double* s, const double* e, double* out) {
  for (int f = 0; f < NW; ++f) out[f] = w[f] + 0.5 * s[f] + e[f];
}
static inline void face_right(const double* w, const double* s, const double* e, double* out) {
  for (int f = 0; f < NW; ++f) out[f] = w[f] - 0.5 * s[f] + e[f];
}

/* One pencil of sweep (muscl.f90:194-215 and the y/z copies): cells 1..n
 * along axis d, addressed through the index callbacks. */
void orc_sweep(const double* w, double* q, const double* evo, const double* s, double dt) {
  const int nx = G.nx, ny = G.ny, nz = G.nz, so = G.secondorder;
  if (nx != 1) {                                      /* muscl.f90:191-216 */
    const double delta = dt * G.dxinv;
#pragma omp parallel for schedule(static) if (nz > 1)
    for (int iz = 1; iz <= nz; ++iz)
      for (int iy = 1; iy <= ny; ++iy) {
        double wl[NW], wr[NW], fl[NF], fr[NF];
        if (so) {
          face_left(&w[iw(0, iy, iz)], &s[is_(1, 0, iy, iz)], &evo[ie(0, iy, iz)], wl);
          face_right(&w[iw(1, iy, iz)], &s[is_(1, 1, iy, iz)], &evo[ie(1, iy, iz)], wr);
        } else {
          memcpy(wl, &w[iw(0, iy, iz)], sizeof wl);
          memcpy(wr, &w[iw(1, iy, iz)], sizeof wr);
        }
        orc_riemann(wl, wr, fr, 1);
        for (int ix = 1; ix <= nx; ++ix) {
          memcpy(fl, fr, sizeof fl);
          if (so) {
            face_left(&w[iw(ix, iy, iz)], &s[is_(1, ix, iy, iz)], &evo[ie(ix, iy, iz)], wl);
            face_right(&w[iw(ix + 1, iy, iz)], &s[is_(1, ix + 1, iy, iz)], &evo[ie(ix + 1, iy, iz)], wr);
          } else {
            memcpy(wl, &w[iw(ix, iy, iz)], sizeof wl);
            memcpy(wr, &w[iw(ix + 1, iy, iz)], sizeof wr);
          }
          orc_riemann(wl, wr, fr, 1);
          orc_integration(fl, fr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
  if (ny != 1) {                                      /* muscl.f90:219-244 */
    const double delta = dt * G.dyinv;
#pragma omp parallel for schedule(static) if (nz > 1)
    for (int iz = 1; iz <= nz; ++iz)
      for (int ix = 1; ix <= nx; ++ix) {
        double wl[NW], wr[NW], fl[NF], fr[NF];
        if (so) {
          face_left(&w[iw(ix, 0, iz)], &s[is_(2, ix, 0, iz)], &evo[ie(ix, 0, iz)], wl);
          face_right(&w[iw(ix, 1, iz)], &s[is_(2, ix, 1, iz)], &evo[ie(ix, 1, iz)], wr);
        } else {
          memcpy(wl, &w[iw(ix, 0, iz)], sizeof wl);
          memcpy(wr, &w[iw(ix, 1, iz)], sizeof wr);
        }
        orc_riemann(wl, wr, fr, 2);
        for (int iy = 1; iy <= ny; ++iy) {
          memcpy(fl, fr, sizeof fl);
          if (so) {
            face_left(&w[iw(ix, iy, iz)], &s[is_(2, ix, iy, iz)], &evo[ie(ix, iy, iz)], wl);
            face_right(&w[iw(ix, iy + 1, iz)], &s[is_(2, ix, iy + 1, iz)], &evo[ie(ix, iy + 1, iz)], wr);
          } else {
            memcpy(wl, &w[iw(ix, iy, iz)], sizeof wl);
            memcpy(wr, &w[iw(ix, iy + 1, iz)], sizeof wr);
          }
          orc_riemann(wl, wr, fr, 2);
          orc_integration(fl, fr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
  if (nz != 1) {                                      /* muscl.f90:247-272 */
    const double delta = dt * G.dzinv;
#pragma omp parallel for schedule(static)
    for (int iy = 1; iy <= ny; ++iy)
      for (int ix = 1; ix <= nx; ++ix) {
        double wl[NW], wr[NW], fl[NF], fr[NF];
        if (so) {
          face_left(&w[iw(ix, iy, 0)], &s[is_(3, ix, iy, 0)], &evo[ie(ix, iy, 0)], wl);
          face_right(&w[iw(ix, iy, 1)], &s[is_(3, ix, iy, 1)], &evo[ie(ix, iy, 1)], wr);
        } else {
          memcpy(wl, &w[iw(ix, iy, 0)], sizeof wl);
          memcpy(wr, &w[iw(ix, iy, 1)], sizeof wr);
        }
        orc_riemann(wl, wr, fr, 3);
        for (int iz = 1; iz <= nz; ++iz) {
          memcpy(fl, fr, sizeof fl);
          if (so) {
            face_left(&w[iw(ix, iy, iz)], &s[is_(3, ix, iy, iz)], &evo[ie(ix, iy, iz)], wl);
            face_right(&w[iw(ix, iy, iz + 1)], &s[is_(3, ix, iy, iz + 1)], &evo[ie(ix, iy, iz + 1)], wr);
          } else {
            memcpy(wl, &w[iw(ix, iy, iz)], sizeof wl);
            memcpy(wr, &w[iw(ix, iy, iz + 1)], sizeof wr);
          }
          orc_riemann(wl, wr, fr, 3);
          orc_integration(fl, fr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
}

/* --------------------------------------------------------- timestep.f90 -- */
/* hydrostep(w), timestep.f90:26-57: returns min(cfl*v, dt_in). */
double orc_hydrostep(const double* w, double dt_in) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  double v = 1e6;
#pragma omp parallel for schedule(static) reduction(min : v) if (nz > 1)
  for (int iy = 1; iy <= ny; ++iy)
    for (int ix = 1; ix <= nx; ++ix)
      for (int iz = 1; iz <= nz; ++iz) {
        const double* c = &w[iw(ix, iy, iz)];
        double a = sqrt(G.g * c[4] / c[0]);
        double vx = G.dx / (fabs(c[1]) + a);
        double vy = G.dy / (fabs(c[2]) + a);
        double vz = G.dz / (fabs(c[3]) + a);
        double m = vx;
        m = fmin2(m, vy);
        m = fmin2(m, vz);
        m = fmin2(m, v);
        v = m;
      }
  double dt = fmin2(G.cfl * v, dt_in);
  if (dt <= 0.0) set_err(EVORA_ERR_DT);
  return dt;
}

/* thermalstep(q,w), timestep.f90:72-104: returns min(conduction limit,
 * dt_in).  pressure(q) resynchronises q in place with dual energy, as the
 * reference's call does. */
double orc_thermalstep(double* q, const double* w, double dt_in) {
  double v = 1e99;
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double* c = &q[iq(ix, iy, iz)];
        double press = orc_pressure(c);
        double temp = press / c[0] * G.temp0;            /* press2temp, comp.f90:87-102 */
        double kappa = G.kappa0 * pow(temp, 2.5);
        v = fmin2(w[iw(ix, iy, iz)] / kappa, v);
      }
  v = G.c_cond * pow(G.dx, 2.0) * v / G.temp0;
  double dt = fmin2(v, dt_in);
  if (dt <= 0.0) set_err(EVORA_ERR_DT);
  return dt;
}

/* coolstep(q,w), timestep.f90:106-143: returns min(dt_in, c_cooldt v), v
 * the smallest cooling time |p / (Gamma - Lambda)| over the cells (from
 * 1e6), with T from w's pressure and the cell's species as they stand.  As
 * in the reference, the equilibrium abundances are computed with module
 * global's nH and nHe (the last cell of the last chem or initchem, not this
 * cell's) and written back into q(7:12): they are the start values of the
 * next chem. */
double orc_coolstep(double* q, const double* w, double dt_in) {
  double v = 1e6;
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double* c = &q[iq(ix, iy, iz)];
        const double press = w[iw(ix, iy, iz) + 4];
        const double temp = press / nsum(c + 6) * G.temp0;     /* press2temp, comp.f90:96-97 */
        double r[9], cr[13], lambda, gamma;
        orc_comprates(temp, r, cr);
        orc_cieabundance(G.nH, G.nHe, c + 6, r);
        orc_cool(c + 6, cr, &lambda, &gamma);
        const double coolio = gamma - lambda;
        const double cooltime = fabs(press / coolio);
        v = fmin2(v, cooltime);
      }
  double dt = fmin2(dt_in, G.c_cooldt * v);
  if (dt <= 0.0) set_err(EVORA_ERR_DT);
  return dt;
}

/* thermalflux, conduction.f90:126-148 (simplekappa) */
static double orc_thermalflux(double templ, double tempr, double deltainv) {
  double kappa_eff = 1.0 / G.g1;
  double dtempdx = (tempr - templ) * deltainv;
  return -(kappa_eff * dtempdx);
}

/* thermalintegration, conduction.f90:150-164 */
static void orc_thermalintegration(double jl, double jr, double* q, double delta) {
  double de = delta * (jl - jr);
  q[4] = q[4] + de;
  q[5] = q[5] + G.g1 * de / pow(q[0], G.g1);
}

static double orc_temp(const double* w) { return w[4] / w[0] * G.temp0; }

/* thermalconduction(q,w), conduction.f90:26-122: sweeps in x, y, z from
 * the same w (ghosts from bound), the interface flux carried along each
 * pencil. */
void orc_thermalconduction(double* q, const double* w, double dt) {
  if (G.nx != 1) {
    double delta = dt * G.dxinv;
    for (int iz = 1; iz <= G.nz; ++iz)
      for (int iy = 1; iy <= G.ny; ++iy) {
        double tempr = orc_temp(&w[iw(1, iy, iz)]);
        double jr = orc_thermalflux(orc_temp(&w[iw(0, iy, iz)]), tempr, G.dxinv);
        for (int ix = 1; ix <= G.nx; ++ix) {
          double jl = jr, templ = tempr;
          tempr = orc_temp(&w[iw(ix + 1, iy, iz)]);
          jr = orc_thermalflux(templ, tempr, G.dxinv);
          orc_thermalintegration(jl, jr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
  if (G.ny != 1) {
    double delta = dt * G.dyinv;
    for (int iz = 1; iz <= G.nz; ++iz)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double tempr = orc_temp(&w[iw(ix, 1, iz)]);
        double jr = orc_thermalflux(orc_temp(&w[iw(ix, 0, iz)]), tempr, G.dyinv);
        for (int iy = 1; iy <= G.ny; ++iy) {
          double jl = jr, templ = tempr;
          tempr = orc_temp(&w[iw(ix, iy + 1, iz)]);
          jr = orc_thermalflux(templ, tempr, G.dyinv);
          orc_thermalintegration(jl, jr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
  if (G.nz != 1) {
    double delta = dt * G.dzinv;
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double tempr = orc_temp(&w[iw(ix, iy, 1)]);
        double jr = orc_thermalflux(orc_temp(&w[iw(ix, iy, 0)]), tempr, G.dzinv);
        for (int iz = 1; iz <= G.nz; ++iz) {
          double jl = jr, templ = tempr;
          tempr = orc_temp(&w[iw(ix, iy, iz + 1)]);
          jr = orc_thermalflux(templ, tempr, G.dzinv);
          orc_thermalintegration(jl, jr, &q[iq(ix, iy, iz)], delta);
        }
      }
  }
}

/* chem(q), chemistry.f90:72-121: pressure() with its dual-energy
 * write-back; with chemistry the CIE species q(7:12) and the cooling over
 * T.dt (cie); the temperature and Jeans pressure floors; E and S corrected
 * by the pressure change when cooling or a floor is on. */
void orc_chem(double* q) {
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double* c = &q[iq(ix, iy, iz)];
        double press = orc_pressure(c);
        double oldpress = press;
        if (G.chemistry) {
          G.nH = G.chiH * c[0];
          G.nHe = G.chiHe * c[0];
          if (G.noncie) orc_ncie(c[0], &press, c + 6);
          else orc_cie(c[0], &press, c + 6);
        }
        if (G.cooling || G.tempfloor || G.jeansfloor) {
          if (G.tempfloor) {
            /* temp2press, comp.f90:104-119 */
            double pfloor = G.chemistry ? G.temp_fl * nsum(c + 6) * G.temp0inv : G.temp_fl * c[0] * G.temp0inv;
            press = fmax2(press, pfloor);
          }
          if (G.jeansfloor) {
            double pfloor = G.jeansfloor0 * c[0] * c[0];
            press = fmax2(press, pfloor);
          }
          double dpress = press - oldpress;
          c[4] = c[4] + dpress * G.g1inv;
          c[5] = c[5] + dpress / pow(c[0], G.g1);
        }
      }
}

/* chem(q) at the time scalars s (dt for the cooling). */
void orc_chem_at(double* q, const double* s) {
  put_time(s);
  orc_chem(q);
}

/* initchem(q), chemistry.f90:26-70: fully neutral. */
void orc_initchem(double* q) {
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double* c = &q[iq(ix, iy, iz)];
        const double nH = G.chiH * c[0], nHe = G.chiHe * c[0];
        G.nH = nH;
        G.nHe = nHe;
        (void)orc_pressure(c);
        for (int i = 7; i <= G.nq; ++i) c[i - 1] = (i == 7) ? nH : (i == 9 ? nHe : kNfloor);
      }
}

/* updatetime(go,dump,k), timestep.f90:147-171, non-comoving branch. */
void orc_updatetime(int* go, double* t, double* dt) {
  if (G.tend - *t <= *dt) {
    *dt = G.tend - *t;
    *go = 0;
  }
  *t = *t + *dt;
}

/* ------------------------------------------------------------- driver -- */
/* The time loop of main.f90:109-203 without gravity, chemistry species and
 * output: hydro, the comoving time scalars (cosmostep, compcosmo,
 * updatetime, compunits), the pressure floors, thermal conduction and the
 * expansion terms when enabled.  Runs until go is cleared, max_steps is
 * reached or an error is raised.  Arrays w, evo, s are scratch of
 * orc_array_sizes() elements, allocated here.  trace (optional) receives 8
 * values per step: the 7 time scalars after updatetime and the dump number
 * the step raised (0: none).  Returns the error mask; *t and *steps report
 * the end state, *dt_last the last step. */
int orc_run_trace(double* q, int max_steps, double* trace, double* t, int* steps, double* dt_last, int* go_out) {
  if (G.noncie) return EVORA_ERR_ARG;   /* the 12-field hydro update is not restated */
  int64_t nq, nw, ne, ns;
  orc_array_sizes(&nq, &nw, &ne, &ns);
  double* w = (double*)calloc((size_t)nw, sizeof(double));
  double* evo = (double*)calloc((size_t)ne, sizeof(double));   /* main.f90:76-77 */
  double* s = (double*)calloc((size_t)ns, sizeof(double));
  if (!w || !evo || !s) {
    free(w); free(evo); free(s);
    return EVORA_ERR_NOMEM;
  }
  int go = 1, k = 0, k4 = 1;
  start_time_();
  orc_err = 0;
  while (go && k < max_steps) {
    orc_primitive(w, q);
    orc_bound(w);
    T.dt = 1e99;
    T.dt = orc_hydrostep(w, T.dt);
    if (G.cooldt) T.dt = orc_coolstep(q, w, T.dt);          /* main.f90:120 */
    if (G.conduction) T.dt = orc_thermalstep(q, w, T.dt);  /* main.f90:121 */
    if (orc_err) break;
    if (G.supercomoving) {                                  /* main.f90:125-128 */
      orc_cosmostep_();
      if (orc_err) break;
      orc_compcosmo_();
    }
    int dump = 0;
    orc_updatetime_(&go, &dump, k4);                        /* main.f90:130 */
    if (orc_err) break;
    if (G.supercomoving) {                                  /* main.f90:132-136 */
      orc_compunits_();
      if (G.chemistry) {
        orc_compbackground_();
        orc_compcoef_();
      }
    }
    if (G.secondorder) orc_compevo(w, evo, s, T.dt);
    orc_sweep(w, q, evo, s, T.dt);
    if (G.chemistry || G.tempfloor || G.jeansfloor) orc_chem(q);   /* main.f90:167 */
    if (G.conduction) {                                     /* main.f90:169-175 */
      orc_primitive(w, q);
      orc_bound(w);
      orc_thermalconduction(q, w, T.dt);
    }
    if (G.supercomoving && !G.atomic) orc_expansion_(q);    /* main.f90:178 */
    if (trace) {
      get_time(trace + 8 * k);
      trace[8 * k + 7] = dump ? k4 : 0;
    }
    if (dump) k4 = k4 + 1;                                  /* main.f90:197-202 */
    ++k;
    if (orc_err) break;
  }
  free(w); free(evo); free(s);
  *steps = k;
  *t = T.t;
  *dt_last = T.dt;
  if (go_out) *go_out = go;
  return orc_err;
}

int orc_run(double* q, int max_steps, double* t, int* steps, double* dt_last, int* go_out) {
  return orc_run_trace(q, max_steps, NULL, t, steps, dt_last, go_out);
}

/* ------------------------------------------------------------------ ICs -- */
/* ic(q) of ic/shocktube.f90:59-100: Riemann problem split at x_diss along
 * direction dir (1..3); coordinates of comp.f90:150-162. */
int orc_ic_shocktube(double* q, double dl, double ul, double pl, double dr, double ur,
                     double pr, double x_diss, int dir) {
  if (dir < 1 || dir > 3) return EVORA_ERR_ARG;
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double x = G.x0 + (double)(ix - 1) * G.dx;
        double y = G.y0 + (double)(iy - 1) * G.dy;
        double z = G.z0 + (double)(iz - 1) * G.dz;
        double d, u, p;
        if ((dir == 1 && x < x_diss) || (dir == 2 && y < x_diss) || (dir == 3 && z < x_diss)) {
          d = dl; u = ul; p = pl;
        } else {
          d = dr; u = ur; p = pr;
        }
        double* c = &q[iq(ix, iy, iz)];
        c[0] = d;
        c[1] = dir == 1 ? d * u : 0.0;
        c[2] = dir == 2 ? d * u : 0.0;
        c[3] = dir == 3 ? d * u : 0.0;
        c[4] = 0.5 * d * (u * u) + p / G.g1;
        c[5] = p / pow(d, G.g1);
      }
  return 0;
}

/* ic(q) of ic/kevinhelmholtz.f90:40-69 (2D shear layer with a localised
 * sinusoidal vy perturbation; pi and the literals 0.1, 0.05 are single
 * precision there, global.f90:98). */
int orc_ic_kh2d(double* q) {
  const double pi = (double)3.1415927f;
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double x = G.x0 + (double)(ix - 1) * G.dx;
        double y = G.y0 + (double)(iy - 1) * G.dy;
        double r = fabs(y - 0.5);
        double d, u;
        if (r <= 0.25) { d = 2.0; u = 0.5; } else { d = 1.0; u = -0.5; }
        double v = (double)0.1f * sin(4 * pi * x) *
                   (exp(-((y - 0.25) * (y - 0.25)) / (double)0.05f) +
                    exp(-((y - 0.75) * (y - 0.75)) / (double)0.05f));
        double p = 2.5;
        double* c = &q[iq(ix, iy, iz)];
        c[0] = d;
        c[1] = d * u;
        c[2] = d * v;
        c[3] = 0;
        c[4] = .5 * d * ((u * u) + (v * v)) + p / (G.g - 1);
        c[5] = p / pow(d, G.g - 1);
      }
  return 0;
}

/* SplitMix64 (Steele, Lea, Flood 2014), the seeded generator of the
 * synthetic 3D Kelvin-Helmholtz workload. */
static uint64_t splitmix64(uint64_t* x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* The 3D Kelvin-Helmholtz workload (no counterpart in the reference's ic/):
 * slab |y - 0.5| < 0.25 with rho = 2, vx = +0.5, outside rho = 1,
 * vx = -0.5, uniform p = 2.5, vz = 0 and
 *   vy = amp * sum_{k=1..4} sin(2 pi k x + phi_k),
 * phi_k = 2 pi u_k with u_k the top 53 bits of successive SplitMix64 draws
 * from `seed`.  Conserved fields as in ic/kevinhelmholtz.f90:61-66. */
int orc_ic_kh3d(double* q, uint64_t seed, double amp) {
  const double twopi = 6.283185307179586;
  double phi[4];
  uint64_t st = seed;
  for (int k = 0; k < 4; ++k) phi[k] = twopi * ((double)(splitmix64(&st) >> 11) * 0x1.0p-53);
  for (int iz = 1; iz <= G.nz; ++iz)
    for (int iy = 1; iy <= G.ny; ++iy)
      for (int ix = 1; ix <= G.nx; ++ix) {
        double x = G.x0 + (double)(ix - 1) * G.dx;
        double y = G.y0 + (double)(iy - 1) * G.dy;
        double d, u;
        if (fabs(y - 0.5) < 0.25) { d = 2.0; u = 0.5; } else { d = 1.0; u = -0.5; }
        double v = 0.0;
        for (int k = 0; k < 4; ++k) v += sin(twopi * (double)(k + 1) * x + phi[k]);
        v = amp * v;
        double p = 2.5;
        double* c = &q[iq(ix, iy, iz)];
        c[0] = d;
        c[1] = d * u;
        c[2] = d * v;
        c[3] = 0.0;
        c[4] = 0.5 * d * ((u * u) + (v * v)) + p / G.g1;
        c[5] = p / pow(d, G.g1);
      }
  return 0;
}
