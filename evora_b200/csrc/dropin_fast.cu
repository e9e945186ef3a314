// Drop-in layer kernels, default arithmetic (FMA contraction allowed).
#define EVORA_NS fast
#include "dropin_kernels.cuh"
#include "dropin_api.h"

namespace evora {
namespace fast {
const DropinOps kOps = {launch_primitive, launch_bound, launch_cfl, launch_compevo, launch_sweep};
}
}  // namespace evora
