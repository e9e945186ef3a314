// dropin_api.h -- the launcher table of the drop-in layer kernels, one
// instance per arithmetic mode (dropin_fast.cu, dropin_strict.cu).
#pragma once

#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace evora {

struct DropinOps {
  // ctl: step control of a resident grid (device memory), or nullptr for a
  // direct call with an explicit dt.
  void (*primitive)(const HydroParams&, double* w, double* q, unsigned* err, const GridCtl* ctl,
                    cudaStream_t);
  void (*bound)(const HydroParams&, double* w, const GridCtl* ctl, cudaStream_t);
  void (*cfl)(const HydroParams&, const double* w, unsigned long long* smax, const GridCtl* ctl,
              cudaStream_t);
  void (*compevo)(const HydroParams&, const double* w, double* evo, double* s, double dt,
                  const GridCtl* ctl, cudaStream_t);
  void (*sweep)(const HydroParams&, const double* w, double* q, const double* evo, const double* s,
                double dt, unsigned* err, const GridCtl* ctl, cudaStream_t);
};

// kOps: the plain build's layouts; kOpsCie: q(12) with species carried (the
// equilibrium-chemistry build); kOpsNcie: q(12) and w(11) with 12 advected
// fields (the non-equilibrium build).
namespace fast { extern const DropinOps kOps, kOpsCie, kOpsNcie; }
namespace strict { extern const DropinOps kOps, kOpsCie, kOpsNcie; }

}  // namespace evora
