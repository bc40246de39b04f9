// Internal interface shared by the stepper and the ensemble.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/spectral_b200.h"
#include "sns_ops.cuh"

namespace sns {

// The caching device pool behind sns_malloc / sns_free.
int pool_malloc(void** ptr, size_t bytes);
int pool_free(void* ptr);

// A stepper of complex fields (sns_ns_create) or of the half spectrum of real
// fields (sns_ns_create_real).
int ns_create(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
              int prec, void* stream, bool real);

// The bootstrap of ns.cpp:132-153 on caller-owned fields: V <- V1, C0 <- cross0,
// with six work fields U.
int ns_bootstrap_fields(Dims d, int prec, double nu, double dt, const void* const V0[3],
                        const void* const omega0[3], void* const V[3], void* const C0[3],
                        void* const U[6], cudaStream_t s);

}  // namespace sns
