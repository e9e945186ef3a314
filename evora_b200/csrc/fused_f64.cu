// Fused backend, FP64 state and arithmetic (FMA contraction allowed).
#define EVORA_FNS f64
#define EVORA_T double
#define EVORA_TX 32
#define EVORA_TY 4
#define EVORA_ZC 32
#include "fused_inst.cuh"
