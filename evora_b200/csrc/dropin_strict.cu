// Drop-in layer kernels, strict arithmetic: this file is compiled with
// --fmad=false so that no multiply-add is contracted, as in a gfortran -O3
// x86-64 build of the reference.
#define EVORA_NS strict
#include "dropin_kernels.cuh"
#include "dropin_api.h"

namespace evora {
namespace strict {
// the plain build (q(6), w(5)), the CIE build (q(12), w(5): species carried,
// not advected) and the non-equilibrium build (q(12), w(11), 12 advected
// fields), global.f90:30-36
const DropinOps kOps = {launch_primitive<EVORA_NQ, EVORA_NW>, launch_bound<EVORA_NW>, launch_cfl<EVORA_NW>,
                        launch_compevo<EVORA_NW>, launch_sweep<EVORA_NQ, EVORA_NW, EVORA_NQ>};
const DropinOps kOpsCie = {launch_primitive<EVORA_NQ_CHEM, EVORA_NW>, launch_bound<EVORA_NW>, launch_cfl<EVORA_NW>,
                           launch_compevo<EVORA_NW>, launch_sweep<EVORA_NQ_CHEM, EVORA_NW, EVORA_NQ>};
const DropinOps kOpsNcie = {launch_primitive<EVORA_NQ_CHEM, 11>, launch_bound<11>, launch_cfl<11>,
                            launch_compevo<11>, launch_sweep<EVORA_NQ_CHEM, 11, EVORA_NQ_CHEM>};
}
}  // namespace evora
