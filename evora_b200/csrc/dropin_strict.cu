// Drop-in layer kernels, strict arithmetic: this file is compiled with
// --fmad=false so that no multiply-add is contracted, as in a gfortran -O3
// x86-64 build of the reference.
#define EVORA_NS strict
#include "dropin_kernels.cuh"
#include "dropin_api.h"

namespace evora {
namespace strict {
const DropinOps kOps = {launch_primitive, launch_bound, launch_cfl, launch_compevo, launch_sweep};
}
}  // namespace evora
