/*
 * harness.c -- TEST INFRASTRUCTURE ONLY.  Drives the mechanical C
 * translation of the reference's Fortran (oracle/_ref/evora_ref.c, made by
 * oracle/ref/f2c.py from the reference sources) the way main.f90 does:
 * namelist values -> compparameter -> decomposition, then the hydro subset
 * of the time loop (main.f90:109-203).  The routines the translation calls
 * but that are not part of the hydro path (cleanstop, MPI broadcasts, the
 * species solvers) are provided here; a Fortran `stop` returns to the caller
 * through longjmp with a nonzero status.
 */
#include <setjmp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/evora_gpu.h"
#if defined(REF_NCIE)
#include "../_ref/evora_ref_ncie.c"  /* the build with -DNONCIE: nq = nf = 12, nw = 11 */
#elif defined(REF_CIE)
#include "../_ref/evora_ref_cie.c"   /* the build with -DCIE: nq = 12 */
#else
#include "../_ref/evora_ref.c"
#endif

static jmp_buf g_jmp;
static int g_armed = 0;

void ref_stop(void) {
  if (g_armed) longjmp(g_jmp, 1);
  abort();
}
void ref_cleanstop(void) { ref_stop(); }
void ref_bcastdouble(double* x) { (void)x; }
void ref_bcastcoef(void) {}
/* the species solvers of chem that this build does not contain */
#ifndef REF_CIE
void ref_cie(double* rho, double* press, double* n) { (void)rho; (void)press; (void)n; ref_stop(); }
/* the plain build has no chemistry coefficients or background to compute */
static void ref_compcoef(void) {}
static void ref_compbackground(void) {}
static void ref_initchem(double* q) { (void)q; ref_stop(); }
#endif
#ifndef REF_NCIE
void ref_ncie(double* rho, double* press, double* n) { (void)rho; (void)press; (void)n; ref_stop(); }
#endif

/* &ic_para of ic/shocktube.f90:39 */
static double nml_dl = 1.0, nml_ul = 0.0, nml_pl = 1.0, nml_dr = 0.125, nml_ur = 0.0, nml_pr = 0.1,
              nml_x_diss = 0.5;
static int nml_dir = 1;
void ref_namelist_ic_para(double* dl, double* ul, double* pl, double* dr, double* ur, double* pr,
                          double* x_diss, int* dir) {
  *dl = nml_dl; *ul = nml_ul; *pl = nml_pl; *dr = nml_dr; *ur = nml_ur; *pr = nml_pr;
  *x_diss = nml_x_diss; *dir = nml_dir;
}

#define GUARD(body)            \
  do {                         \
    if (setjmp(g_jmp)) {       \
      g_armed = 0;             \
      return 1;                \
    }                          \
    g_armed = 1;               \
    body;                      \
    g_armed = 0;               \
  } while (0)

/* readparameter defaults (parameter.f90:41-82) for the namelist variables
 * that compparameter and decomposition read, then the hydro subset from p;
 * a single rank (startstop.f90:59-63 with mpisize = 1). */
int ref_setup_c(const evora_params* p) {
  G_iconly = 0; G_hydro = 1;
  G_secondorder = p->secondorder; G_solver = p->solver; G_limiter = p->limiter;
  G_cfl = p->cfl; G_g = p->g; G_atomic = p->atomic;
  G_nx = p->nx; G_ny = p->ny; G_nz = p->nz;
  G_xmin = p->xmin; G_xmax = p->xmax; G_ymin = p->ymin; G_ymax = p->ymax;
  G_zmin = p->zmin; G_zmax = p->zmax;
  G_boundtype = p->boundtype;
  G_gravity = 0;
  G_tstart = p->tstart; G_tend = p->tend;
  G_supercomoving = p->supercomoving; G_c_cosmo = p->c_cosmo; G_omega0 = p->omega0; G_lambda0 = p->lambda0;
  G_hubble0 = p->hubble0; G_box = p->box; G_zstart = p->zstart; G_zend = p->zend;
  for (int i = 0; i < EVORA_NDUMP; ++i) G_dump_redshift[i] = p->dump_redshift[i];
  G_chemistry = p->chemistry; G_noncie = p->noncie; G_cooling = p->cooling; G_background = p->background;
  G_bg = p->bg; G_j0 = p->j0; G_c_chem = p->c_chem; G_substep = p->substep; G_rhoh = p->rhoh;
  G_rhohe = p->rhohe; G_cooldt = p->cooldt; G_c_cooldt = p->c_cooldt;
  if (!G_chemistry) { G_background = 0; G_cooling = 0; }   /* parameter.f90:98-103 */
  if (!G_cooling) G_cooldt = 0;
  G_uv = 0.0;
  G_conduction = p->conduction; G_simplekappa = p->simplekappa; G_c_cond = p->c_cond;
  G_tempfloor = p->tempfloor; G_temp_fl = p->temp_fl; G_jeansfloor = p->jeansfloor; G_c_jeans = p->c_jeans;
  G_fb = p->fb;
  G_dualenergy = p->dualenergy; G_de_thresh = p->de_thresh;
  G_mpisize = 1; G_mpirank = 0; G_master = 1; G_parallel = 0;
  G_local_x_start = 0; G_local_nx = p->nz;
  /* the time scalars a fresh program starts with (static storage) */
  G_dt = 0.0; G_redshift = 0.0; G_oldcosmo = 0.0; G_cosmodot = 0.0; G_expand = 0.0;
  G_nh = 0.0; G_nhe = 0.0;
  /* main.f90:52-62: compparameter, cosmostart (comoving), compunits */
  GUARD(ref_compparameter(); ref_decomposition(); if (G_supercomoving) ref_cosmostart(); ref_compunits();
        if (G_chemistry) { G_chih = G_rhoh / G_mh; G_chihe = G_rhohe / G_mhe; ref_compcoef(); });
  return 0;
}

/* The time scalars (evora_time's order) and the units of module global. */
void ref_get_time_c(double* s) {
  s[0] = G_t; s[1] = G_dt; s[2] = G_cosmo; s[3] = G_oldcosmo; s[4] = G_cosmodot; s[5] = G_expand;
  s[6] = G_redshift;
}
static void put_time(const double* s) {
  G_t = s[0]; G_dt = s[1]; G_cosmo = s[2]; G_oldcosmo = s[3]; G_cosmodot = s[4]; G_expand = s[5];
  G_redshift = s[6];
}
void ref_get_units_c(double* u) { u[0] = G_temp0; u[1] = G_temp0inv; u[2] = G_kappa0; }

int ref_cosmostep_c(double* s) { put_time(s); GUARD(ref_cosmostep()); ref_get_time_c(s); return 0; }
int ref_compcosmo_c(double* s) { put_time(s); GUARD(ref_compcosmo()); ref_get_time_c(s); return 0; }
int ref_updatetime_cosmo_c(int* go, int* dump, int k, double* s) {
  put_time(s);
  GUARD(ref_updatetime(go, dump, &k));
  ref_get_time_c(s);
  return 0;
}
int ref_settime_c(double* s) {
  put_time(s);
  GUARD(ref_compunits(); if (G_supercomoving && G_background) ref_compbackground();
        if (G_supercomoving && G_chemistry) ref_compcoef());
  return 0;
}
int ref_peebles_c(double* s, double* f) { put_time(s); GUARD(ref_peebles(f)); return 0; }
int ref_expansion_c(double* q, double* s) { put_time(s); GUARD(ref_expansion(q)); return 0; }

void ref_sizes_c(int64_t* nq, int64_t* nw, int64_t* ne, int64_t* ns) {
  *nq = (int64_t)G_nq * G_nx * G_ny * G_nz;
  *nw = (int64_t)G_nw * (G_nx + 4) * (G_ny + 4) * (G_nz + 4);
  *ne = (int64_t)G_nw * (G_nx + 2) * (G_ny + 2) * (G_nz + 2);
  *ns = (int64_t)G_nw * 3 * (G_nx + 2) * (G_ny + 2) * (G_nz + 2);
}

void ref_derived_c(double* out) {
  double v[] = {G_g, G_g1, G_g1inv, G_gg1, G_cfl, G_de_thresh1, G_dx, G_dy, G_dz,
                G_dxinv, G_dyinv, G_dzinv, G_x0, G_y0, G_z0, G_volume};
  memcpy(out, v, sizeof v);
}

int ref_primitive_c(double* w, double* q) { GUARD(ref_primitive(w, q)); return 0; }
int ref_bound_c(double* w) { GUARD(ref_bound(w)); return 0; }
int ref_hydrostep_c(double* w, double* dt) {
  G_dt = *dt;
  GUARD(ref_hydrostep(w));
  *dt = G_dt;
  return 0;
}
int ref_updatetime_c(int* go, double* t, double* dt) {
  int dump = 0, k4 = 1;
  G_t = *t; G_dt = *dt;
  GUARD(ref_updatetime(go, &dump, &k4));
  *t = G_t; *dt = G_dt;
  return 0;
}
int ref_compevo_c(double* w, double* evo, double* s, double dt) {
  G_dt = dt;
  GUARD(ref_compevo(w, evo, s));
  return 0;
}
int ref_sweep_c(double* w, double* q, double* evo, double* s, double dt) {
  G_dt = dt;
  GUARD(ref_sweep(w, q, evo, s));
  return 0;
}

int ref_chem_c(double* q) { GUARD(ref_chem(q)); return 0; }
int ref_chem_at_c(double* q, double* s) { put_time(s); GUARD(ref_chem(q)); return 0; }
int ref_initchem_c(double* q) { GUARD(ref_initchem(q)); return 0; }
/* coef(13, 2) as [13][2] rows, then uv */
void ref_get_coef_c(double* out) {
  for (int i = 0; i < 13; ++i)
    for (int j = 0; j < 2; ++j) out[2 * i + j] = G_coef[i + 13 * j];
  out[26] = G_uv;
}
int ref_thermalstep_c(double* q, double* w, double* dt) {
  G_dt = *dt;
  GUARD(ref_thermalstep(q, w));
  *dt = G_dt;
  return 0;
}
/* coolstep(q,w), timestep.f90:106-143: reads the module's nH and nHe as the
 * last chem or initchem left them and writes the abundances back into q. */
int ref_coolstep_c(double* q, double* w, double* dt) {
#ifdef REF_CIE
  G_dt = *dt;
  GUARD(ref_coolstep(q, w));
  *dt = G_dt;
  return 0;
#else
  (void)q; (void)w; (void)dt;
  return 1;
#endif
}
int ref_thermalconduction_c(double* q, double* w, double dt) {
  G_dt = dt;
  GUARD(ref_thermalconduction(q, w));
  return 0;
}

/* main.f90:109-203 without gravity or output: hydro and, when enabled, the
 * cooling time-step limit (120, chemistry build), the comoving time scalars
 * (125-136), chem with the species and the pressure floors (167), thermal
 * conduction (121, 169-175) and the expansion terms (178).  trace
 * (optional): 8 values per step, the time scalars after updatetime and the
 * dump number the step raised. */
int ref_run_trace_c(double* q, int max_steps, double* trace, double* t, int* steps, double* dt, int* go_out) {
  int64_t nq, nw, ne, ns;
  ref_sizes_c(&nq, &nw, &ne, &ns);
  double* w = calloc((size_t)nw, sizeof(double));
  double* evo = calloc((size_t)ne, sizeof(double));
  double* s = calloc((size_t)ns, sizeof(double));
  int go = 1, dump = 0, k = 0, k4 = 1, rc = 0;
  G_t = G_tstart;
  G_cosmo = 1.0; G_oldcosmo = 0.0; G_cosmodot = 0.0; G_expand = 0.0; G_redshift = 0.0;
  if (setjmp(g_jmp)) {
    g_armed = 0;
    rc = 1;
    goto done;
  }
  g_armed = 1;
  if (G_supercomoving) ref_cosmostart();
  ref_compunits();
  G_uv = 0.0;
  if (G_chemistry) ref_compcoef();   /* initchem's coefficients (main.f90:94) */
  while (go && k < max_steps) {
    ref_primitive(w, q);
    ref_bound(w);
    G_dt = 1e99;
    if (G_hydro) ref_hydrostep(w);
#ifdef REF_CIE
    if (G_cooldt) ref_coolstep(q, w);
#endif
    if (G_conduction) ref_thermalstep(q, w);
    if (G_supercomoving) {
      ref_cosmostep();
      ref_compcosmo();
    }
    ref_updatetime(&go, &dump, &k4);
    if (G_supercomoving) {   /* main.f90:132-136 */
      ref_compunits();
      if (G_background) ref_compbackground();
      if (G_chemistry) ref_compcoef();
    }
    if (G_secondorder) ref_compevo(w, evo, s);
    if (G_hydro) ref_sweep(w, q, evo, s);
    if (G_chemistry || G_tempfloor || G_jeansfloor) ref_chem(q);
    if (G_conduction) {
      ref_primitive(w, q);
      ref_bound(w);
      ref_thermalconduction(q, w);
    }
    if (G_supercomoving && !G_atomic) ref_expansion(q);
    if (trace) {
      ref_get_time_c(trace + 8 * k);
      trace[8 * k + 7] = dump ? k4 : 0;
    }
    if (dump) {
      dump = 0;
      k4 = k4 + 1;
    }
    k = k + 1;
  }
  g_armed = 0;
done:
  *t = G_t;
  *dt = G_dt;
  *steps = k;
  if (go_out) *go_out = go;
  free(w); free(evo); free(s);
  return rc;
}

int ref_ic_shocktube_c(double* q, double dl, double ul, double pl, double dr, double ur, double pr,
                       double x_diss, int dir) {
  nml_dl = dl; nml_ul = ul; nml_pl = pl; nml_dr = dr; nml_ur = ur; nml_pr = pr;
  nml_x_diss = x_diss; nml_dir = dir;
  GUARD(ref_ic_shocktube(q));
  return 0;
}
int ref_ic_kh_c(double* q) { GUARD(ref_ic_kevinhelmholtz(q)); return 0; }
int ref_riemann_c(double* wl, double* wr, double* f, int dir) {
  GUARD(ref_riemannsolver(wl, wr, f, &dir));
  return 0;
}

int ref_run_c(double* q, int max_steps, double* t, int* steps, double* dt, int* go_out) {
  return ref_run_trace_c(q, max_steps, NULL, t, steps, dt, go_out);
}
