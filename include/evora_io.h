/* evora_io.h -- the reference's file formats for the hydro state.
 *
 * Dump files (write.f90:26-65), unit files (units.f90:76-159), in-run
 * snapshots (snapshot.f90:196-360) and the cuts and slices of the
 * post-processor (post.f90:85-246, comp.f90:201-239), written byte for byte
 * as the reference writes them (gfortran conventions for unformatted record
 * markers and formatted edit descriptors).  The evora_grid_* variants read
 * the state from the device: a snapshot gathers the two planes it prints
 * (and, for the brick-of-values files, one FP32 density and temperature per
 * cell computed on the device) instead of the whole grid.
 *
 * All functions return 0 or an evora_status bit (EVORA_ERR_IO for file
 * errors, EVORA_ERR_ARG for bad sizes, EVORA_ERR_PRESSURE where the
 * reference's pressure() would stop, comp.f90:74-84).
 */
#ifndef EVORA_IO_H
#define EVORA_IO_H

#include <stdint.h>

#include "evora_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ dump files -- */
/* writedata (write.f90:47-65): a Fortran unformatted sequential file with
 * two records, each framed by 4-byte little-endian length markers:
 *   [nn, nx, ny, nz, lz, mz] (int32) and q(nn, nx, ny, lz:mz) (FP64,
 *   column-major, the whole array of one rank).
 * A rank's slab holds z planes lz..mz; a single-process run has lz = 1 and
 * mz = nz.  Records longer than 2^31 - 9 bytes are refused (EVORA_ERR_ARG):
 * gfortran splits those into subrecords, which this writer does not. */
int evora_write_dump(const char* path, const double* q, int32_t nn, int32_t nx, int32_t ny, int32_t nz,
                     int32_t lz, int32_t mz);

/* opendata (write.f90:179-214): reads the header record only. */
int evora_read_dump_header(const char* path, int32_t header[6]);

/* opendata + `read (10) q` (post.f90:183-186): the header and the array;
 * `capacity` is the number of doubles q can hold (nn*nx*ny*(mz-lz+1) are
 * read).  Record markers are checked. */
int evora_read_dump(const char* path, int32_t header[6], double* q, int64_t capacity);

/* ----------------------------------------------------------------- units -- */
/* The unit scales of module global (units.f90:26-73) as the unit file lists
 * them (units.f90:92-109). */
typedef struct evora_units {
  double t, cosmo, redshift, length0, time0, density0, velocity0, temp0, press0, number0, chem0, photo0,
      cool0, heat0, jeans0, jeansfloor0, kappa0, meanfreepath0;
} evora_units;

/* compunits (units.f90:26-73) for a run without comoving coordinates
 * (cosmo = 1, redshift = 0, jeans floor off): g is the adiabatic index as
 * the parameter file gives it, fb the baryon fraction (default 1). */
void evora_units_noncomoving(double t, double g, double fb, evora_units* u);

/* compunits (units.f90:26-73), both branches, for the parameters p at the
 * time state s (t, cosmo, redshift; NULL = tstart, a = 1, z = 0): with
 * supercomoving the cosmological units at expansion factor a (h =
 * hubble0/100, d0 = omega0 rhoc h^2, t0 = 1/H0, l0 = box Mpc/h), and the
 * Jeans floor jeansfloor0 = (dx / jeans0 / c_jeans)^2 when it is on.  g is
 * the gas constant after compparameter (5/3 with atomic).  EVORA_ERR_ARG for
 * parameters compparameter rejects. */
int evora_compunits(const evora_params* p, const evora_time* s, evora_units* u);

/* writeunits (units.f90:76-113) and readunits (units.f90:115-159). */
int evora_write_units(const char* path, const evora_units* u);
int evora_read_units(const char* path, evora_units* u);

/* ------------------------------------------------------------- snapshots -- */
enum evora_snapshot_what {
  EVORA_SNAP_CUT = 1,   /* <k3>.x and (not 1D) <k3>.x0   snapshot.f90:236-276 */
  EVORA_SNAP_SLICE = 2, /* <k3>.xy and <k3>.xz           snapshot.f90:279-314 */
  EVORA_SNAP_BOV = 4    /* <k3>.{dens,temp}.bov{,data}   snapshot.f90:225-228, 317-341, write.f90:66-104 */
};

/* snapshot(k3, q) (snapshot.f90:196-360) from a host q(nq, nx, ny, nz) into
 * directory `dir` (the reference's "snap/"); nq = 6, or 12 with chemistry,
 * whose temperatures are p / sum(q(7:12)) temp0 (press2temp, comp.f90:
 * 87-102).  Like the reference, pressure() runs on every printed cell and,
 * with dualenergy, resynchronises that cell's E or S in q (comp.f90:60-69).
 * The .xz slice is opened in append mode, as in the reference. */
int evora_snapshot(const evora_params* p, double* q, const evora_units* u, int32_t k3, int32_t what,
                   const char* dir);

/* The same from a grid's device-resident state, at the grid's time t:
 * gathers the z = max(nz/2,1) and y = max(ny/2,1) planes for cuts and
 * slices and computes the FP32 density and temperature bricks on the device
 * (with chemistry: the whole q(12) through the host writer); with
 * dualenergy the resynchronised cells are written back to the grid, as the
 * reference's in-place pressure() calls leave them. */
int evora_grid_snapshot(evora_grid* g, const evora_units* u, int32_t k3, int32_t what, const char* dir);

/* One plane of the grid's state in the reference layout (FP64, 6 values per
 * cell, lower remaining axis fastest): axis 1 = the x plane ix = index,
 * 2 = the y plane iy = index, 3 = the z plane iz = index (1-based).  `out`
 * holds 6 * (cells of the plane) doubles, host or device memory. */
int evora_grid_get_plane(evora_grid* g, int32_t axis, int32_t index, double* out);
int evora_grid_set_plane(evora_grid* g, int32_t axis, int32_t index, const double* in);

/* ---------------------------------------------------------- post-process -- */
/* `post cs <infile>` (post.f90:85-246): reads <datadir>/<infile>.000,
 * .001, ... (the ranks' z slabs, until one ends at nz), computes the state
 * vector of comp.f90:201-239 on the middle lines and planes and writes
 * <outdir>/<infile>.{x,y,z,xy,xyz}.cut and .{xy,xz,yz}.slice as the
 * reference does (including its writing of the diagonal cut's data into the
 * .xyz file, post.f90:228).  Hydro build: q(6) dumps, 12 values per cell.
 * With chemistry (the CIE build): q(12) dumps, 26 values: also the species
 * per density and the number densities and, with cooling, Lambda and Gamma
 * from the rates at the cell's T (rates.f90's own powers), with the
 * coefficients of compbackground and compcoef at the units of the dump
 * (post.f90:58-62); cieabundance leaves the cell's species in equilibrium,
 * as in the reference.  p gives the grid and gas of the run (the reference
 * rereads them from data/parameter), fb the baryon fraction, u the unit
 * scales of the dump (data/<infile>.units). */
int evora_cuts_and_slices(const evora_params* p, double fb, const evora_units* u, const char* datadir,
                          const char* infile, const char* outdir);

#ifdef __cplusplus
}
#endif

#endif /* EVORA_IO_H */
