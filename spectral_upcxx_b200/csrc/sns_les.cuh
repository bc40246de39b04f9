// Eddy-viscosity (LES) extension of the fused NS step (host interface).
#pragma once

#include <cuda_runtime.h>

#include "sns_ns.cuh"

namespace sns {

enum ClosureModel : int { CLOSURE_NONE = 0, CLOSURE_SMAGORINSKY = 1, CLOSURE_MLP = 2 };

struct Closure {
  int model = CLOSURE_NONE;
  double csd2 = 0;            // Smagorinsky (Cs Delta)^2
  const void* mlp = nullptr;  // packed MLP (device), CLOSURE_MLP
};

constexpr int kLESWork = 12;  // work fields of the closure step
constexpr int kLESLaunches = 5;

// One step with the eddy-viscosity term of `cl` (the plain step when
// cl.model == CLOSURE_NONE is ns_step_once): V, C0 as in ns_step_once, U
// holds kLESWork fields, stats as in ns_step_once.
// Takes (reads and clears) the record of a tensor-core wait of the closure's
// x pass that ran out; synchronises the device.
int les_tc_status_take(int* timed_out);
int les_step_once(const NSPlan& pl, void* const V[3], void* const C0[3], void* const U[kLESWork],
                  double* stats, double nu, double dt, const Closure& cl, cudaStream_t s);

}  // namespace sns
