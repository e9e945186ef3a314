// Fused backend, FP64, strict arithmetic: compiled with --fmad=false so that
// the result equals a gfortran -O3 x86-64 build of the reference bit for bit
// on rho, m and E (the entropy field goes through pow).
#define EVORA_FNS f64s
#define EVORA_T double
#define EVORA_FAST 0
#define EVORA_PRECISION_F32 0
#include "fused_inst.cuh"
