/*
 * evora_gpu.h -- C ABI of the B200 (sm_100a) hydro update of evora.
 *
 * The hot path of the reference is the hydro update that main.f90 drives
 * once per step (main.f90:109-155):
 *
 *     call primitive(w,q)      muscl.f90:26-43   (q2w/pressure, comp.f90:26-85)
 *     call bound(w)            boundary.f90:26-113
 *     dt = 1d99
 *     call hydrostep(w)        timestep.f90:26-57
 *     call updatetime(go,..)   timestep.f90:147-171
 *     call compevo(w,evo,s)    muscl.f90:45-113  (comp_slope 115-169)
 *     call sweep(w,q,evo,s)    muscl.f90:171-274 (riemann.f90, integration)
 *
 * This header offers two layers over the same CUDA kernels:
 *
 *  1. The drop-in layer (evora_primitive ... evora_sweep): one entry point per
 *     reference subroutine, same arguments, same array layouts (column-major
 *     AoS, field index fastest, ghost frames as allocated in main.f90:72-75).
 *     Parameters that the Fortran code reads from `module global` are set
 *     once with evora_set_params(); time-step scalars are passed explicitly.
 *     Array pointers may be device pointers (used in place) or host pointers
 *     (staged through device buffers on every call).
 *
 *  2. The resident layer (evora_grid_*): the whole step fused on the device,
 *     state kept in HBM across steps in structure-of-arrays form, FP64 or
 *     FP32 arithmetic.  This is the fast path a driver uses between dumps.
 *
 * All entry points return a status: 0 on success, otherwise a bit mask of
 * EVORA_ERR_* codes.  The reference prints a message and stops at each of
 * these conditions; the library reports them and leaves the decision to the
 * caller.  No entry point traps, and no device wait is unbounded.
 */
#ifndef EVORA_GPU_H
#define EVORA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
enum evora_status {
  EVORA_OK = 0,
  EVORA_ERR_PRESSURE = 1,         /* p <= 0 recovering primitives, comp.f90:74-84 */
  EVORA_ERR_RIEMANN_PRESSURE = 2, /* wl(5)<=0 or wr(5)<=0, riemann.f90:61-66,111-116 */
  EVORA_ERR_HLL = 4,              /* no HLL branch taken, riemann.f90:87-90 */
  EVORA_ERR_HLLC = 8,             /* no HLLC branch taken, riemann.f90:148-150 */
  EVORA_ERR_DT = 16,              /* hydro step <= 0, timestep.f90:51-55 */
  EVORA_ERR_LIMITER = 32,         /* unknown slope limiter, muscl.f90:164-167 */
  EVORA_ERR_SOLVER = 64,          /* unknown Riemann solver, riemann.f90:38-41 */
  EVORA_ERR_ARG = 128,            /* invalid argument, size or call order */
  EVORA_ERR_CUDA = 256,           /* CUDA runtime error (see evora_last_error) */
  EVORA_ERR_NOMEM = 512,          /* device allocation failed */
  EVORA_ERR_TIMEOUT = 1024,       /* a bounded host or device wait gave up */
  EVORA_ERR_IO = 2048,            /* a file could not be opened, written or read */
  EVORA_ERR_COSMO = 4096,         /* timestepiteration did not converge, timestep.f90:220-223 */
  EVORA_ERR_CHEM = 8192           /* abundances out of range (ncheck, chemistry.f90:159-176),
                                     no or no converging electron-density root (cie.f90:131-134,
                                     164-167), or a cooling update that does not end */
};

/* Number of conserved / primitive / flux fields of the plain build
 * (global.f90:35: nq=6, nf=6, nw=5).  Field order of q: rho, rho*u, rho*v,
 * rho*w, E, S = p/rho^(g-1); of w: rho, u, v, w, p. */
#define EVORA_NQ 6
#define EVORA_NW 5
/* Length of dump_redshift (global.f90:137: ndump = 100). */
#define EVORA_NDUMP 100

/* ------------------------------------------------------------ parameters -- */
/* The hydro subset of namelist &para (parameter.f90:30-37). */
typedef struct evora_params {
  int32_t nx, ny, nz;   /* cells per axis; ny = nz = 1 is 1D, nz = 1 is 2D   */
  int32_t solver;       /* 1 = HLL, 2 = HLLC                                 */
  int32_t limiter;      /* 1 = minmod, 2 = monotonised central, 3 = van Leer */
  int32_t boundtype;    /* 1 = zero gradient, 2 = periodic,
                           3 = zero gradient with reflecting upper x face    */
  int32_t secondorder;  /* Fortran logical: MUSCL-Hancock predictor on       */
  int32_t dualenergy;   /* Fortran logical: dual-energy pressure recovery    */
  int32_t atomic;       /* Fortran logical: forces g = 5.0/3.0 (single prec) */
  int32_t gravity;      /* Fortran logical: self-gravity after each hydro
                           step (gravitation.f90, non-comoving branch)      */
  double g, cfl, de_thresh;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double tstart, tend;
  int32_t conduction;   /* Fortran logical: explicit thermal conduction after
                           each step (conduction.f90) and its time-step
                           limit (thermalstep, timestep.f90:72-104)         */
  int32_t simplekappa;  /* Fortran logical: conductivity 1/(g-1); the other
                           branch reads unset variables in the reference's
                           plain build and is refused (EVORA_ERR_ARG)       */
  double c_cond;        /* conduction time-step factor                      */
  int32_t tempfloor;    /* Fortran logical: pressure floor at temp_fl after
                           each step (chem, chemistry.f90:92-121)           */
  int32_t jeansfloor;   /* Fortran logical: pressure floor jeansfloor0 rho^2 */
  double temp_fl;       /* temperature of the floor                         */
  double c_jeans;       /* Jeans floor factor (units.f90:66-71)             */
  double fb;            /* baryon fraction (units: jeans0 = sqrt(pi g fb))  */
  /* comoving coordinates (cosmology.f90; main.f90:58, 124-136, 178, 184-185) */
  int32_t supercomoving;  /* Fortran logical: expansion factor a(t) integrated
                             with the step, comoving units, the expansion
                             terms (unless atomic) and the comoving source
                             of gravity                                      */
  double c_cosmo;         /* expansion time-step factor (cosmostep)          */
  double omega0, lambda0; /* density and cosmological-constant parameters    */
  double hubble0, box;    /* H0 in km/s/Mpc; box size in Mpc/h (units)       */
  double zstart, zend;    /* first and last redshift                         */
  double dump_redshift[EVORA_NDUMP]; /* redshifts of the intermediate dumps,
                             in the order they are reached; -1 = unused      */
  /* chemistry and cooling of the CIE build (chemistry.f90, cie.f90,
   * rates.f90; main.f90:94, 135, 167): with chemistry the state is
   * q(12, nx, ny, nz), q(7:12) = n(H, H+, He, He+, He++, e-) in equilibrium
   * (not advected: the CIE build's fluxes are nf = 6, global.f90:31-32).
   * The non-equilibrium build (noncie: ncie.f90's Patankar solver, the
   * species advected, nf = 12, nw = 11) is accepted by the drop-in
   * routines (the hydro routines on the q(12)/w(11) layout, evora_chem,
   * evora_initchem); grids, evora_hydrostep_noalloc and evora_coolstep
   * refuse it (EVORA_ERR_ARG).                                               */
  int32_t chemistry;      /* Fortran logical                                 */
  int32_t noncie;         /* Fortran logical: non-equilibrium species (ncie) */
  int32_t cooling;        /* Fortran logical: radiative cooling (cie)         */
  int32_t background;     /* Fortran logical: UV background (implicitcie)     */
  int32_t bg;             /* background model 1..3 (compbackground)           */
  int32_t cooldt;         /* Fortran logical: cooling time-step limit        */
  double j0;              /* background intensity                            */
  double c_chem, substep; /* cooling sub-cycle factors (cie.f90:41)           */
  double rhoh, rhohe;     /* H and He mass fractions                          */
  double c_cooldt;        /* cooling time-step factor                         */
} evora_params;

/* The chemistry build's layout: EVORA_NQ_CHEM values per cell in q. */
#define EVORA_NQ_CHEM 12

/* The derived constants of compparameter (parameter.f90:164-265) that the
 * hydro path reads from module global. */
typedef struct evora_derived {
  double g, g1, g1inv, gg1, cfl, de_thresh1;
  double dx, dy, dz, dxinv, dyinv, dzinv;
  double x0, y0, z0, volume;
  int32_t onedimension, twodimension;
} evora_derived;

/* Defaults of readparameter (parameter.f90:41-82).  Note g = 1.4 and the
 * other defaults there are single-precision literals: g is stored as
 * (double)1.4f = 1.39999997615814..., as the reference does. */
void evora_params_default(evora_params* p);

/* compparameter (parameter.f90:164-265), hydro subset.  Returns
 * EVORA_ERR_ARG for non-positive sizes, EVORA_ERR_SOLVER /
 * EVORA_ERR_LIMITER for unknown options (riemann.f90:38-41,
 * muscl.f90:164-167 stop at first use; here they are checked up front). */
int evora_compparameter(const evora_params* p, evora_derived* d);

/* Element counts of the reference arrays for the given grid (main.f90:72-75):
 *   q(nq, nx, ny, nz), w(nw, nx+4, ny+4, nz+4), evo(nw, nx+2, ny+2, nz+2),
 *   s(nw, 3, nx+2, ny+2, nz+2).  The ghost frames exist in every axis, also
 *   for 1D and 2D grids, as in the reference. */
void evora_array_sizes(const evora_params* p, int64_t* nq_elems, int64_t* nw_elems,
                       int64_t* nevo_elems, int64_t* ns_elems);

/* Last CUDA error string seen by the library (static storage). */
const char* evora_last_error(void);

/* Library version string. */
const char* evora_version(void);

/* Self-test of the FP64 reciprocal and square root of the fast arithmetic
 * forms (no counterpart in the reference, which divides and calls sqrt): for
 * host arrays x[n], out[i] = the device's fast reciprocal of x[i],
 * out[n + i] = the device's correctly rounded 1.0 / x[i], out[2n + i] = the
 * fast square root and out[3n + i] = the correctly rounded sqrt(x[i]); out
 * holds 4n doubles. */
int evora_selftest_rcp(const double* x, double* out, int64_t n);

/* Self-test of the arithmetic the default mode's chem(q) uses (no
 * counterpart in the reference, which calls exp and divides): for host
 * arrays x[n], out[i] = the table-driven exp(x[i]) (Tang's method),
 * out[n + i] = the Newton-refined reciprocal of x[i] and out[2n + i] = the
 * hardware's approximate reciprocal it starts from; out holds 3n doubles. */
int evora_selftest_exp(const double* x, double* out, int64_t n);

/* -------------------------------------------------------- drop-in layer -- */
/* Set the module-global hydro parameters used by the routines below (the
 * analogue of `use global` after compparameter).  Must be called first. */
int evora_set_params(const evora_params* p);

/* Arithmetic mode of the drop-in layer: 0 = default (contracted FMAs), 1 =
 * strict (no FMA contraction; matches a gfortran -O3 x86-64 build of the
 * reference bit for bit where libm is not involved). */
int evora_set_strict(int32_t strict);

/* Resident mode of the drop-in layer (no reference counterpart: the
 * reference's arrays live in host memory).  With mode EVORA_RESIDENT_FP64
 * (the arithmetic of evora_set_strict) or EVORA_RESIDENT_FP32 (the FP32
 * form), the routines that main.f90:109-155 calls keep the fluid state on
 * the GPU between calls instead of copying the host arrays in and out:
 *   evora_primitive(w, q)  binds host array q to a resident grid, uploading it
 *                          when it is new or was invalidated; w is not written
 *   evora_bound(w), evora_compevo(w, evo, s, dt)   nothing to do (the ghost
 *                          map, slopes and predictor run inside the update)
 *   evora_hydrostep(w, dt) dt from the CFL maxima of the resident state; it
 *                          also reports p <= 0 (which primitive reports
 *                          without residency)
 *   evora_sweep(w, q, evo, s, dt)  enqueues the fused update with this dt;
 *                          errors it raises are returned by the next
 *                          hydrostep or evora_sync
 * Host q is brought up to date only by evora_sync(q), and automatically
 * before any other drop-in routine or file writer takes q (those that
 * change q make the next evora_primitive upload it again).  w, evo and s are
 * never written in this mode.  0 ends the mode after copying the state back.
 * The results equal the non-resident routines' (bit for bit in strict FP64). */
enum evora_resident_mode { EVORA_RESIDENT_FP64 = 1, EVORA_RESIDENT_FP32 = 2 };
int evora_set_resident(int32_t mode);

/* Resident mode: copies the resident state of host array q back into q (no
 * reference counterpart; call it before the driver reads q, e.g. before
 * evolution, snapshot and writedump, main.f90:191-206).  No-op for arrays
 * that are not resident. */
int evora_sync(double* q);

/* Resident mode: the caller changed host q itself; the next evora_primitive
 * uploads it again (no reference counterpart). */
int evora_invalidate(const double* q);

/* primitive(w,q), muscl.f90:26-43.  w interior <- q2w(q) for every cell.
 * With dualenergy the routine writes back q(5) or q(6) (comp.f90:60-72). */
int evora_primitive(double* w, double* q);

/* bound(w), boundary.f90:26-113.  Fills the two ghost layers of w: x faces,
 * then y faces, then z faces, each over the full ghost-inclusive extent. */
int evora_bound(double* w);

/* hydrostep(w), timestep.f90:26-57.  *dt = min(cfl * v, *dt) with
 * v = min(1e6, min over interior cells of dx_d / (|u_d| + a)).
 * Returns EVORA_ERR_DT if the result is <= 0. */
int evora_hydrostep(const double* w, double* dt);

/* A variant of evora_hydrostep that allocates nothing (no counterpart in the
 * reference).  For callers that may not call cudaMalloc: a driver that
 * allocates all device memory at start-up and none inside its time loop, or
 * code running while a memory pool owns the device or other work is being
 * captured.  Same arithmetic and result as evora_hydrostep, bit for bit.
 * Differences: w must be device memory (no staging copy is made); the
 * reduction scratch is a fixed file-scope device array (about 1.5 MB, held by
 * every GPU that loads the library until exit), which limits the grid to
 * nx*ny*nz <= 16777216 interior cells -- larger grids return EVORA_ERR_ARG
 * with a message in evora_last_error().  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU (concurrent host threads or
 * streams) race on it.  Synchronous: returns after dt is known. */
int evora_hydrostep_noalloc(const double* w, double* dt);

/* thermalstep(q,w), timestep.f90:72-104 (conduction on, simplekappa):
 * dt = min(c_cond dx^2 min(rho / (kappa0 T^2.5)) / temp0, dt) with T from
 * pressure(q) (which resynchronises q in place with dual energy, as the
 * reference's call does) and rho from w.  EVORA_ERR_DT if dt <= 0,
 * EVORA_ERR_ARG unless conduction and simplekappa are set. */
int evora_thermalstep(double* q, const double* w, double* dt);

/* coolstep(q,w), timestep.f90:106-143 (chemistry with cooling and cooldt):
 * dt = min(dt, c_cooldt v), v the smallest cooling time |p / (Gamma -
 * Lambda)| over the cells (from 1e6), T = w(5) / sum(n) temp0 with the
 * cell's abundances q(7:12) as they stand, the rates at the coefficients
 * evora_settime (or evora_set_params) computed.  As in the reference, the
 * equilibrium abundances this computes are written back into q(7:12), and
 * they use the n(H), n(He) of module global as the last evora_chem or
 * evora_initchem left them (its last cell's), not the cell's own.
 * EVORA_ERR_DT if dt <= 0, EVORA_ERR_CHEM for abundances out of range,
 * EVORA_ERR_ARG unless cooldt is set. */
int evora_coolstep(double* q, const double* w, double* dt);

/* thermalconduction(q,w), conduction.f90:26-122 (simplekappa): the x, y
 * and z conduction sweeps over dt from the primitives w (ghosts filled by
 * bound), updating E and S of q in place. */
int evora_thermalconduction(double* q, const double* w, double dt);

/* chem(q), chemistry.f90:72-121: pressure() with its dual-energy
 * write-back; with chemistry (q(12, ...)) the CIE abundances q(7:12) and,
 * with cooling, the pressure advanced over dt by the sub-cycled cooling
 * update (cie.f90:26-56; dt and, comoving, the units and UV background from
 * evora_settime), or with noncie the abundances advanced over dt by ncie's
 * Patankar sub-cycles (ncie.f90:26-149), with the same cooling update; then the temperature floor (tempfloor: press = max(press,
 * temp_fl rho / temp0), or temp_fl sum(n) / temp0 with chemistry) and the
 * Jeans floor (jeansfloor: press = max(press, jeansfloor0 rho^2)), with E and
 * S corrected by the pressure change when cooling or a floor is on. */
int evora_chem(double* q);

/* initchem(q), chemistry.f90:26-70, on a host q(12, nx, ny, nz) (the
 * chemistry build's layout): fully neutral species, n(H) = rho rhoH / mH,
 * n(He) = rho rhoHe / mHe, the others at nfloor = 1e-40; pressure() runs on
 * every cell as there (resynchronising E or S with dual energy).
 * EVORA_ERR_ARG without chemistry or for a device pointer. */
int evora_initchem(double* q);

/* gravpotential(q,phi), gravitation.f90:26-53: the potential of the
 * density of q (FFT Poisson solve with the reference's discrete Green's
 * function), from the source 4 pi G (rho - mean rho), or with supercomoving
 * a (3/2 omega0) (rho / fb - 1) with a from evora_settime.  phi is the
 * reference's complex(8) phi(nx,ny,nz) (interleaved re, im); the imaginary
 * part is written as 0. */
int evora_gravpotential(const double* q, double* phi);

/* gravintegration(q,phi,...), gravitation.f90:170-243, for one process:
 * the gravitational source terms of m and E over dt from the real part of
 * phi (periodic centred differences). */
int evora_gravintegration(double* q, const double* phi, double dt);

/* updatetime(go,dump,k), timestep.f90:147-171, non-comoving branch:
 * if tend - t <= dt then dt = tend - t, go = false; then t = t + dt.
 * dump and k are accepted for signature parity (they only matter in the
 * supercomoving branch: evora_updatetime_cosmo). */
int evora_updatetime(int32_t* go, int32_t* dump, int32_t* k, double* t, double* dt);

/* The time scalars of module global (global.f90:86) that the reference
 * broadcasts after each time step (bcasttime, parallel.f90:71-95), plus
 * oldcosmo and cosmodot. */
typedef struct evora_time {
  double t, dt;
  double cosmo;      /* expansion factor a (1 without comoving coordinates) */
  double oldcosmo;   /* a before the last compcosmo                         */
  double cosmodot;   /* da/dt                                               */
  double expand;     /* a da/dt                                             */
  double redshift;   /* 1/a - 1                                             */
} evora_time;

/* The comoving time routines of cosmology.f90 and timestep.f90 on the host
 * (scalar work; the resident layer runs the same arithmetic on the device):
 *   evora_cosmostart    cosmostart (cosmology.f90:26-36): t = tstart,
 *                       redshift = zstart, a = 1/(1+zstart), da/dt; without
 *                       supercomoving a = 1 (compparameter) and the rest 0
 *   evora_cosmostep     cosmostep (timestep.f90:59-70):
 *                       dt = min(a / (da/dt) c_cosmo, dt); EVORA_ERR_DT if <= 0
 *   evora_compcosmo     compcosmo (cosmology.f90:38-51): a advanced over dt by
 *                       the reference's Runge-Kutta step (rungekutta,
 *                       cosmology.f90:136-163, including its last stage at
 *                       the unadvanced a), then da/dt, expand, redshift
 *   evora_updatetime_cosmo  updatetime (timestep.f90:147-171), both branches;
 *                       with supercomoving the step is shortened onto zend
 *                       (go = false) or onto dump_redshift(k) (dump = true)
 *                       by timestepiteration (timestep.f90:173-226);
 *                       EVORA_ERR_COSMO if that does not converge.
 * Parameters come from evora_set_params. */
int evora_cosmostart(evora_time* s);
int evora_cosmostep(evora_time* s);
int evora_compcosmo(evora_time* s);
int evora_updatetime_cosmo(int32_t* go, int32_t* dump, int32_t* k, evora_time* s);

/* peebles(fpeebles), cosmology.f90:76-97: the linear growth rate
 * d ln D / d ln a at s->cosmo, by the reference's trapezoid rule (steps of
 * 1e-8 in a from 1e-8).  The cosmological initial conditions scale their
 * Zel'dovich velocities with it (ic/cosmo.f90:91-92, ic/pancake.f90:65-66). */
int evora_peebles(const evora_time* s, double* fpeebles);

/* Set the time scalars the drop-in routines read from module global: dt and
 * expand for evora_expansion, a for the comoving source of
 * evora_gravpotential, and (with supercomoving) the units that depend on a
 * (compunits, units.f90:26-73: temp0 for the floors of evora_chem and for
 * conduction, kappa0).  The reference recomputes them after every
 * compcosmo (main.f90:132-136). */
int evora_settime(const evora_time* s);

/* expansion(q), cosmology.f90:53-72: for every cell, pressure(q) (with its
 * dual-energy write-back), then E -= dt (3g-5) expand p / (g-1) and
 * S -= dt (3g-5) expand S, with dt and expand from evora_settime.  main.f90
 * calls it after conduction when supercomoving and not atomic. */
int evora_expansion(double* q);

/* compevo(w,evo,s), muscl.f90:45-113, with comp_slope (115-169).
 * Fills the slopes s and the half-step predictor evo over the interior plus
 * one ghost layer, using the step size dt. */
int evora_compevo(const double* w, double* evo, double* s, double dt);

/* sweep(w,q,evo,s), muscl.f90:171-274.  Updates q in place with the x, y
 * and z flux differences of each cell, in that order (integration,
 * muscl.f90:276-290), using one Riemann solve per interface. */
int evora_sweep(const double* w, double* q, const double* evo, const double* s, double dt);

/* ------------------------------------------------------- resident layer -- */
typedef struct evora_grid evora_grid;
typedef struct evora_multigrid evora_multigrid;

enum evora_precision { EVORA_FP64 = 0, EVORA_FP32 = 1 };

enum evora_grid_flags {
  /* Carry the entropy field S = q(6) (as the reference does).  Without this
   * flag only rho, m, E are advanced: S never feeds back into them when
   * dualenergy is off, so rho, m, E are unchanged bit for bit. */
  EVORA_CARRY_ENTROPY = 1,
  /* Strict arithmetic (no FMA contraction) for FP64 grids. */
  EVORA_STRICT = 2,
  /* Run the step with the drop-in layer's per-routine kernels on
   * device-resident arrays in the reference layouts (FP64 only), instead of
   * the fused kernel.  Slower; kept as the reference-shaped device path. */
  EVORA_REFERENCE_KERNELS = 4
};

/* Creates a grid on the current CUDA device.  Allocates the resident state
 * (two copies of the conserved fields plus a few scalars). */
int evora_grid_create(const evora_params* p, int32_t precision, int32_t flags,
                      evora_grid** out);
int evora_grid_destroy(evora_grid* g);

/* As evora_grid_create, but all device memory of the grid is allocated
 * stream-ordered on `stream` (cudaMallocAsync from the device's default
 * pool) and freed the same way by evora_grid_destroy, so creating and
 * destroying grids never synchronises the device; the grid works on that
 * stream for its whole life.  For callers that create and retire many grids
 * while others run (a request loop). */
int evora_grid_create_async(const evora_params* p, int32_t precision, int32_t flags, void* stream,
                            evora_grid** out);

/* Work on this CUDA stream (cudaStream_t); NULL = the default stream. */
int evora_grid_set_stream(evora_grid* g, void* stream);

/* Load / read back the conserved state in the reference layout
 * q(6, nx, ny, nz) (column-major, field fastest).  Host or device pointer.
 * set_q also resets t = tstart, k = 0, go = true and the status word. */
int evora_grid_set_q(evora_grid* g, const double* q);
int evora_grid_get_q(evora_grid* g, double* q);

/* Advances up to nsteps steps of the reference loop (main.f90:109-155):
 * primitive, bound, hydrostep, updatetime, compevo, sweep.  Stops early when
 * updatetime clears go.  Asynchronous: returns after enqueueing, unless a
 * status check is requested with sync != 0, in which case it waits for the
 * stream and returns the accumulated error mask. */
int evora_grid_step(evora_grid* g, int32_t nsteps, int32_t sync);

/* Time, last step size, go flag and step count (synchronises the stream). */
int evora_grid_time(evora_grid* g, double* t, double* dt, int32_t* go, int64_t* k);

/* The grid's time scalars (synchronises the stream), and the dump the last
 * step raised: with supercomoving, a step that updatetime shortened onto
 * dump_redshift(k) sets *dump = k (1-based; the reference then writes dump
 * number k, main.f90:197-202), otherwise *dump = 0.  While a dump is
 * pending the grid does not step; this call clears it. */
int evora_grid_cosmo(evora_grid* g, evora_time* s, int32_t* dump);

/* Accumulated device error mask (synchronises the stream). */
int evora_grid_status(evora_grid* g);

/* Sums of q(1..6) over the interior in FP64 (the totals of evolution,
 * snapshot.f90:159-193, before the multiplication by the cell volume). */
int evora_grid_totals(evora_grid* g, double out[6]);

/* ------------------------------------------------ multi-grid batches -- */
/* Many resident 2D and 3D grids of uneven sizes advanced together (no
 * counterpart in the reference, which runs one grid per process).  Each step
 * of all member grids is three launches: one control kernel (every grid's
 * hydrostep and updatetime, timestep.f90:26-57, 147-171, with its own dt and
 * t), one persistent update launch whose CTAs pull (grid, tile) work items
 * from a queue (largest first) and run the fused update of muscl.f90:171-290
 * on them, and one closing control kernel; steps are replayed from CUDA
 * graphs.  A member's results equal those of the grid stepped alone (bit for
 * bit).  Members share precision and flags, are 2D or 3D, and carry no
 * physics after the update (gravity, conduction, floors, chemistry,
 * comoving coordinates): EVORA_ERR_ARG otherwise.  While a grid is a member
 * it is stepped only through its batch; set_q, get_q, time and status work
 * between batch steps, after a step with sync or evora_multigrid_status.
 * The batch works on `stream` (NULL: the default stream). */
int evora_multigrid_create(int32_t precision, int32_t flags, void* stream, evora_multigrid** out);
/* Releases the batch (its member grids stay, stepped alone again). */
int evora_multigrid_destroy(evora_multigrid* m);
int evora_multigrid_add(evora_multigrid* m, evora_grid* g);
int evora_multigrid_remove(evora_multigrid* m, evora_grid* g);
/* Advances every member nsteps steps (members whose run has ended, or that
 * raised an error, pass their state through unchanged).  Asynchronous unless
 * sync != 0. */
int evora_multigrid_step(evora_multigrid* m, int32_t nsteps, int32_t sync);
/* Waits for the batch and reports, in member order, up to max members: the
 * grid, its go flag, its error mask and its step count; *n = members
 * reported. */
int evora_multigrid_status(evora_multigrid* m, evora_grid** grids, int32_t* go, uint32_t* err, int64_t* k,
                           int32_t max, int32_t* n);

/* Tile autotuner (no counterpart in the reference): times every tile shape
 * of the fused update kernel (`reps` launches each) on the grid's own state
 * and keeps the fastest.  The state and the time of the grid are unchanged.
 * ms_per_tile (optional, max_tiles entries) receives the timings. */
int evora_grid_autotune(evora_grid* g, int32_t reps, int32_t* chosen, double* ms_per_tile,
                        int32_t max_tiles);
/* Selects a tile shape by index (0 = the default); a shape that cannot run
 * the grid falls back to 0.  EVORA_FP32_PAIR_TILE is the FP32 table's
 * two-cells-per-thread kernel (packed f32x2; grids of whole 32x8 tiles with
 * 5 fields, HLLC, minmod and the second-order scheme). */
enum { EVORA_FP32_PAIR_TILE = 5 };
int evora_grid_set_tile(evora_grid* g, int32_t tile);

/* Kernel timing (no counterpart in the reference): when on, every step
 * records CUDA events around its CFL kernel, its update kernel and the
 * physics after the update (gravity, floors, conduction, expansion) on the
 * grid's stream.  evora_grid_timing synchronises, returns the summed event
 * times in ms (update_ms: the update and the physics after it), the number
 * of timed steps and the number of kernels the grid launched since timing
 * was switched on, and clears the record; evora_grid_timing_split returns
 * the update and the physics separately. */
int evora_grid_set_timing(evora_grid* g, int32_t on);
int evora_grid_timing(evora_grid* g, double* update_ms, double* cfl_ms, int64_t* steps,
                      int64_t* launches);
int evora_grid_timing_split(evora_grid* g, double* cfl_ms, double* update_ms, double* physics_ms,
                            int64_t* steps, int64_t* launches);

/* ------------------------------------------------------- batched tubes -- */
/* No counterpart in the reference (a one-run CLI): many independent 1D
 * tubes (ny = nz = 1), each a run of the reference loop main.f90:109-155 on
 * its own grid, with its own length n[i], time, step size and end time, all
 * sharing the options of *p (solver, limiter, boundtype, secondorder, g,
 * cfl, xmin/xmax, tstart, tend).  One persistent kernel launch advances every
 * unfinished tube; each CTA stages a whole tube in shared memory and runs its
 * steps there.  Tubes are independent: a tube's result does not depend on the
 * others (bit for bit), and a tube that raises an error stops alone. */
typedef struct evora_batch evora_batch;

int evora_batch_create(const evora_params* p, int32_t ntubes, const int32_t* n, int32_t precision,
                       int32_t flags, evora_batch** out);
int evora_batch_destroy(evora_batch* b);
/* A capturable (non-default) stream; the batch owns one until this is set. */
int evora_batch_set_stream(evora_batch* b, void* stream);
/* q in the reference layout q(6, n[tube]); tube = -1: all tubes concatenated.
 * Host or device pointer.  (Re)starts the tube(s): t = tstart, k = 0. */
int evora_batch_set_q(evora_batch* b, int32_t tube, const double* q);
int evora_batch_get_q(evora_batch* b, int32_t tube, double* q);
/* Per-tube end time (default p->tend); takes effect at the next set_q/run. */
int evora_batch_set_tend(evora_batch* b, int32_t tube, double tend);
/* Advances every running tube by up to max_steps steps (<= 0: until each
 * reaches its end time), in one launch replayed from a CUDA graph cached per
 * step budget.  With sync, waits and returns the OR of the tubes' errors. */
int evora_batch_run(evora_batch* b, int32_t max_steps, int32_t sync);
/* Tube state; returns the tube's error mask.  status: 0 running, 1 done,
 * 2 stopped by an error, 3 idle (no state loaded). */
int evora_batch_info(evora_batch* b, int32_t tube, double* t, double* dt, int32_t* go, int64_t* k,
                     int32_t* status);
/* Total cell-updates done by the batch so far. */
int evora_batch_steps_done(evora_batch* b, int64_t* cell_updates);
/* Threads per CTA (128, 256, 512) and CTAs per SM the shared-memory staging
 * is sized for (tubes longer than that capacity run from global memory). */
int evora_batch_configure(evora_batch* b, int32_t threads, int32_t ctas_per_sm);
/* Autotuner: times every (threads, CTAs per SM) candidate for `steps` steps
 * on the batch's own state (restored after each trial) and keeps the fastest. */
int evora_batch_autotune(evora_batch* b, int32_t steps, int32_t* threads, int32_t* ctas_per_sm);

/* ------------------------------------------------------------- serving -- */
/* No counterpart in the reference (one simulation per process): a request
 * loop with continuous batching.  A request is an initial state q(6, nx, ny,
 * nz) (reference layout, host memory, copied at submit), a grid size and an
 * end time; the other options come from *base.  evora_server_tick admits
 * pending requests in arrival order while their device footprint fits the
 * HBM budget (1D requests also need a free tube slot and arena room), then
 * advances everything admitted by one round -- a time quantum: a grid of c
 * cells gets min(8 * steps_per_tick, steps_per_tick * 2^20 / c) steps, the
 * tube launch up to 8 * steps_per_tick steps per tube: 1D requests
 * together in one persistent batched-tube launch, 2D/3D requests as resident
 * grids on their own streams, concurrently; finished requests are read back
 * and their time to solution (submit to read-back) recorded.  A request's
 * result does not depend on what else is in flight.  One host thread drives
 * a server. */
typedef struct evora_server evora_server;

int evora_server_create(const evora_params* base, int32_t precision, int32_t flags, double hbm_budget_bytes,
                        int32_t steps_per_tick, int32_t max_tube_cells, int32_t max_tubes,
                        evora_server** out);
int evora_server_destroy(evora_server* s);
/* Queues a request; *id identifies it.  boundtype 1..3 overrides the
 * server's for this request (0 keeps it).  EVORA_ERR_ARG if it can never fit. */
int evora_server_submit(evora_server* s, int32_t nx, int32_t ny, int32_t nz, double tend, int32_t boundtype,
                        const double* q0, int64_t* id);
/* As evora_server_submit, without a copy before the call returns: the
 * server's copy threads read q0 after it, so q0 must stay valid and
 * unchanged until the request is no longer pending (evora_server_result
 * reports it running, done or failed).  With q_out (the request's size in
 * the reference layout) the result is copied into q_out before the request
 * reports done or failed; q_out must stay valid until then, and
 * evora_server_result with that same pointer delivers it without a copy.
 * The host copies then overlap the device's rounds. */
int evora_server_submit_borrowed(evora_server* s, int32_t nx, int32_t ny, int32_t nz, double tend,
                                 int32_t boundtype, const double* q0, double* q_out, int64_t* id);
/* One scheduling round (admit, step, retire); reports active/pending counts. */
int evora_server_tick(evora_server* s, int32_t* n_active, int32_t* n_pending);
/* state: 0 pending, 1 running, 2 done, 3 failed, -1 unknown id.  When done or
 * failed and q_out is given, copies the final state (reference layout),
 * latency and step count, and forgets the request.  Returns its error mask. */
int evora_server_result(evora_server* s, int64_t id, double* q_out, double* latency_s, int64_t* steps,
                        int32_t* state);
/* Host seconds spent per round phase so far: out[0] launch, [1] read-back,
 * [2] admission, [3] waiting for the device, [4] freeing, [5] completion
 * checks; out[6] the number of rounds. */
int evora_server_profile(evora_server* s, double out[7]);
/* Device time so far of the rounds' tube launches and of the multi-grid
 * batch's steps (CUDA events around them on their streams), ms. */
int evora_server_device_ms(evora_server* s, double* tube_ms, double* batch_ms);
/* Ids of requests finished (done or failed) since the last call, oldest
 * first, at most max_ids of them; *n receives the count. */
int evora_server_completed(evora_server* s, int64_t* ids, int32_t max_ids, int32_t* n);
/* p50 / p99 time to solution of completed requests, their count, the total
 * cell-updates and the time from the first submit to the last completion. */
int evora_server_stats(evora_server* s, double* p50_s, double* p99_s, int64_t* completed,
                       int64_t* cell_updates, double* span_s);

#ifdef __cplusplus
}
#endif

#endif /* EVORA_GPU_H */
