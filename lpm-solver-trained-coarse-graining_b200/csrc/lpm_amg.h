// Aggregation-AMG preconditioner and the FP32 PCG that uses it (amg.cu): internal declarations.
#pragma once
#include <cstdint>

#include "../../include/lpm_b200.h"
#include "lpm_kernels.h"

struct lpm_amg;  // opaque handle of the C ABI, defined in amg.cu

namespace lpm {

// FP32 AMG-preconditioned CG on the handle's batch: K_ff x = b from x = 0 for every system, b and x (nsys, N, 3)
// FP32 device arrays.  Stop rule, checking interval, per-system tolerances and outputs as cg_solve.
int amg_pcg(lpm_amg* h, const float* b, float* x, const lpm_cg_opts& o, int* iters, double* relres, int* status,
            cudaStream_t st);

// True when the handle was created for this lattice and batch shape and has been set up.
bool amg_matches(const lpm_amg* h, const Lattice& L, const Batch& bt);

}  // namespace lpm
