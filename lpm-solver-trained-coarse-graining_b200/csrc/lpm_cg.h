// Internal declarations of the batched CG engine and the mixed-precision driver.
#pragma once
#include <cstddef>

#include "../../include/lpm_b200.h"
#include "lpm_kernels.h"

namespace lpm {

// Per-system scalar state of a batched CG solve (all device arrays of length nsys unless noted).
struct CgScalars {
    double* part;      // (3, nsys, nblk) per-block partials of up to three inner products
    unsigned* cnt;     // (nsys) last-block counters (start at 0, re-armed by the last block)
    double* bn;        // |b|
    double* rz;        // (2, nsys) r.z of the current / next iteration (ping-pong by iteration parity)
    double* rr;        // r.r of the last completed iteration
    double* pAp;       // p.Ap of the current iteration (written by the operator epilogue)
    double* beta;      // beta of the current iteration
    int* act;          // 1 while a system iterates
    unsigned* nconv;   // (1) systems that left the active set
    int* iters;        // caller output
    double* relres;    // caller output
    int* status;       // caller output
    int nblk;          // partial blocks per system of the vector kernels
};

size_t cg_workspace_bytes(const Lattice& L, int nsys, int precision, int precond);
size_t ir_workspace_bytes(const Lattice& L, int nsys, int precond);

template <typename T>
int cg_solve(const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt, const T* Minv,
             const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws, size_t ws_bytes,
             int* iters, double* relres, int* status, cudaStream_t st);

int ir_solve(const Lattice& L, const double* Kn64, const double* Tv64, const CoefLayout& cl64, const float* Kn32,
             const float* Tv32, const CoefLayout& cl32, const float* Minv32, const Batch& bt, const uint8_t* mask,
             const double* b, double* x, const lpm_ir_opts& o, void* ws, size_t ws_bytes, int* iters,
             double* relres, int* status, int* outer, cudaStream_t st);

}  // namespace lpm
