// CG engine on the TMA-fed SC operator (full boxes, packed (set, 18, n) coefficients): shared scalar state.
#pragma once
#include "lpm_cg.h"

namespace lpm {

// Scalars of the fused CG engine (device arrays of length nsys unless noted).
struct FcgScalars {
    int nsys;
    double* bn;
    double* rz;  // (2, nsys) ping-pong by iteration parity
    double* rr;
    double* pAp;
    double* alpha;
    double* beta;
    int* act;
    unsigned* nconv;
    int* iters;
    double* relres;
    int* status;
    int* itp;  // device copy of the current iteration number (1-based), advanced by the p-update kernel; lets a
               // captured block of iterations replay without host-side parameters
    const double* tols;  // optional per-system tolerance (replaces the scalar tol)
};

// alpha step of system s, run by the last block of the operator epilogue once p.Ap is complete.
__device__ __forceinline__ void cg_alpha_step(const FcgScalars& sc, int s, double pAp, int it)
{
    if (sc.itp) it = *sc.itp;
    sc.pAp[s] = pAp;
    if (!sc.act[s]) {
        sc.alpha[s] = 0.0;
        return;
    }
    const double rzc = sc.rz[((it - 1) & 1) * sc.nsys + s];
    if (!isfinite(pAp) || pAp < 0.0 || !isfinite(rzc)) {
        sc.alpha[s] = 0.0;
        sc.act[s] = 0;
        sc.iters[s] = it;
        sc.status[s] = LPM_STATUS_BREAKDOWN;
        atomicAdd(sc.nconv, 1u);
        return;
    }
    sc.alpha[s] = pAp != 0.0 ? rzc / pAp : 0.0;
}

// beta step of system s in a PCG whose preconditioner output z comes from an operator epilogue (AMG): run by the
// last block once r.z is complete.  Iteration 0 is the initial preconditioner application (beta = 0).
__device__ __forceinline__ void cg_beta_step(const FcgScalars& sc, int s, double rz, int it)
{
    if (sc.itp) it = *sc.itp;
    if (!sc.act[s]) return;
    const double rzo = sc.rz[((it + 1) & 1) * sc.nsys + s];
    sc.rz[(it & 1) * sc.nsys + s] = rz;
    if (!isfinite(rz)) {
        sc.beta[s] = 0.0;
        sc.act[s] = 0;
        sc.iters[s] = it;
        sc.status[s] = LPM_STATUS_BREAKDOWN;
        atomicAdd(sc.nconv, 1u);
        return;
    }
    sc.beta[s] = it > 0 && rzo != 0.0 ? rz / rzo : 0.0;
}

// Batched (P)CG on the TMA operator (dim 3, full box, packed coefficients, tma_supported(nx)).
template <typename T>
int cg_solve_fused(const Lattice& L, const T* Kn, const T* Tv, const Batch& bt, const T* Minv, const uint8_t* mask,
                   const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws, size_t ws_bytes, int* iters,
                   double* relres, int* status, cudaStream_t st);
size_t cg_fused_workspace_bytes(const Lattice& L, int nsys, int rhs_per_set, int elem_bytes, int precond);

}  // namespace lpm
