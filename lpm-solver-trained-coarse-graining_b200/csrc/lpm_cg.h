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
    int* itp;          // device copy of the current iteration number, advanced by the p-update kernel
    const double* tols;  // optional per-system tolerance (replaces the scalar tol)
};

// Optional CUDA-event timing of the operator launches of a solve (prof != nullptr).  prof[0] += ms and prof[1] += count
// over all launches; prof[2] += ms and prof[3] += count over the launches issued while no system had yet left the
// active set (as last seen by the host), i.e. launches that did the full batch's work.  Events are recorded on the
// solve's stream and read back at the host synchronisation points of the loop.
class KmvTimer {
  public:
    KmvTimer(double* prof, cudaStream_t st) : prof_(prof), st_(st)
    {
        if (!prof_) return;
        for (int j = 0; j < kPairs; ++j) {
            cudaEventCreate(&a_[j]);
            cudaEventCreate(&b_[j]);
        }
    }
    ~KmvTimer()
    {
        if (!prof_) return;
        for (int j = 0; j < kPairs; ++j) {
            cudaEventDestroy(a_[j]);
            cudaEventDestroy(b_[j]);
        }
    }
    void begin(bool full)
    {
        if (!prof_) return;
        if (n_ == kPairs) collect();
        full_[n_] = full;
        cudaEventRecord(a_[n_], st_);
    }
    void end()
    {
        if (!prof_) return;
        cudaEventRecord(b_[n_], st_);
        ++n_;
    }
    void collect()  // call after the stream reached the last recorded event
    {
        if (!prof_ || n_ == 0) return;
        if (cudaEventSynchronize(b_[n_ - 1]) != cudaSuccess) return;
        for (int j = 0; j < n_; ++j) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a_[j], b_[j]);
            prof_[0] += ms;
            prof_[1] += 1.0;
            if (full_[j]) {
                prof_[2] += ms;
                prof_[3] += 1.0;
            }
        }
        n_ = 0;
    }

  private:
    static constexpr int kPairs = 64;
    double* prof_;
    cudaStream_t st_;
    cudaEvent_t a_[kPairs], b_[kPairs];
    bool full_[kPairs];
    int n_ = 0;
};

size_t cg_workspace_bytes(const Lattice& L, const Batch& bt, int precision, int precond);
size_t ir_workspace_bytes(const Lattice& L, const Batch& bt, int precond);

template <typename T>
int cg_solve(const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt, const T* Minv,
             const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws, size_t ws_bytes,
             int* iters, double* relres, int* status, cudaStream_t st);

// Persistent engine (cg_persist.cu): one cooperative launch per solve.  persist_fits: the batch has a team shape on
// this device; persist_auto: LPM_ENGINE_AUTO picks it (small batches).  cg_solve routes to it by opts.engine.
// Sets the bound of one team-barrier wait of the persistent engine (ns, process-wide); returns the previous bound.
unsigned long long persist_wait_limit(unsigned long long ns);
bool persist_fits(const Lattice& L, const Batch& bt);
bool persist_auto(const Lattice& L, const Batch& bt, int elem_bytes);
size_t persist_workspace_bytes(const Lattice& L, const Batch& bt, int elem_bytes);
template <typename T>
int cg_solve_persist(const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                     const T* Minv, const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o,
                     void* ws, size_t ws_bytes, int* iters, double* relres, int* status, cudaStream_t st);

// amg != nullptr: the inner solver is the AMG-preconditioned FP32 PCG of the handle (Kn32, Tv32, Minv32 unused).
int ir_solve(const Lattice& L, const double* Kn64, const double* Tv64, const CoefLayout& cl64, const float* Kn32,
             const float* Tv32, const CoefLayout& cl32, const float* Minv32, const Batch& bt, const uint8_t* mask,
             const double* b, double* x, const lpm_ir_opts& o, void* ws, size_t ws_bytes, int* iters,
             double* relres, int* status, int* outer, cudaStream_t st, lpm_amg* amg = nullptr);

}  // namespace lpm
