// Fused backend, FP32 state, slopes and fluxes (compiled with fast
// division/square root); FP64 for the pressure recovery of cells with
// kin > E/2, for the CFL reduction and for the conserved totals.
#define EVORA_FNS f32
#define EVORA_T float
#define EVORA_FAST 1
#define EVORA_PRECISION_F32 1
#include "fused_inst.cuh"
