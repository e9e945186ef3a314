// Fused backend, FP64 state and arithmetic (FMA contraction allowed).
#define EVORA_FNS f64
#define EVORA_T double
#define EVORA_FAST 1
#define EVORA_PRECISION_F32 0
#include "fused_inst.cuh"
