// common.h -- host-side helpers shared by the ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/evora_gpu.h"
#include "hydro_math.cuh"

namespace evora {

// Records a CUDA error for evora_last_error().
void set_cuda_error(cudaError_t e, const char* where);

// evora_params -> validated HydroParams (+ derived constants).
bool params_to_hydro(const evora_params* p, HydroParams* P, evora_derived* d, int* status);

// True for device or managed memory.
bool is_device_pointer(const void* ptr);

// Records a message for evora_last_error().
void set_error_message(const char* msg);

// The module-global parameters set by evora_set_params (false if unset),
// with the units of the time state evora_settime last set.
bool dropin_params(HydroParams* P);

struct CosmoTime;

// The time scalars of the drop-in layer (evora_set_params: the start of the
// run; then evora_settime).  False if no parameters are set.
bool dropin_time(CosmoTime* s);

struct ChemCoef;

// The chemistry's rate coefficients of the drop-in layer (evora_set_params:
// the start of the run; evora_settime with comoving coordinates).
bool dropin_coef(ChemCoef* k);

// Module global's nH, nHe of the drop-in layer: 0 after evora_set_params,
// then the last cell's of each evora_initchem or evora_chem with chemistry
// (chemistry.f90:50-51, 90-91); coolstep reads them.
void dropin_set_nh(double nH, double nHe);
bool dropin_nh(double* nH, double* nHe);

// t = tstart and cosmo = 1 (compparameter), then cosmostart with
// supercomoving (main.f90:52-58).
void start_time(const evora_params* p, const HydroParams& P, CosmoTime* s);

// The parameters a grid was created with.
const evora_params* grid_params(const evora_grid* g);

// The drop-in layer's resident mode drives a fused-backend grid one routine
// at a time.  grid_cfl_maxima: the per-axis maxima of |u_d| + a of the
// current state (from the previous update when it reduced them, else from
// the CFL kernel) into smax on the host; returns the grid's error word.
// grid_update_dt: the fused update of the current state with the caller's
// dt; with sync, waits for it and returns the grid's error word, else only
// enqueues it (launch errors are returned).
int grid_cfl_maxima(evora_grid* g, double smax[3]);
int grid_update_dt(evora_grid* g, double dt, bool sync);

// evora_grid_set_q / evora_grid_get_q without their final wait: the copies
// and conversions are only enqueued on the grid's stream.  q must stay valid
// (set_q) and is complete (get_q) once that stream has been synchronised.
int grid_set_q_async(evora_grid* g, const double* q);
int grid_get_q_async(evora_grid* g, double* q);

// Host arrays q bound to the resident mode's grid: before a routine that
// reads q on the host, the newer device state is copied back
// (dropin_resident_read); before one that also writes it, the device copy is
// then marked stale so that the next evora_primitive uploads q again
// (dropin_resident_write).  No-ops for other pointers or with residency off.
void dropin_resident_read(const double* q);
void dropin_resident_write(const double* q);

// Per cell FP32 density and temperature of the grid's state into host
// arrays of nx*ny*nz values (snapshot.f90:317-341); returns 0, an error
// status of pressure(), or EVORA_ERR_CUDA.
int grid_bov(evora_grid* g, double temp0, float* dens, float* temp);

}  // namespace evora
