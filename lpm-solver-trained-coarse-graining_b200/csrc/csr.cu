// Assembled-matrix solve behind the coarse2d/lin2d.py:166-180 (solve_disp) call site: K_ff x_f = b_f on a CSR
// matrix by Jacobi-preconditioned CG in FP64, all on the device.
//
// The reference factors K[free][:, free] with SuperLU and back-substitutes.  Here the full K stays as the caller
// assembled it (CSR, int64 row pointers, int32 columns, FP64 values) and the free set enters as a per-row mask: with
// p zero on fixed rows, mask(K p) is K_ff p_f.  One iteration is three kernels, each grid-striding over rows with a
// fixed grid so that the per-block partial sums (and with them every scalar) are deterministic:
//   1. k_csr_spmv:  Ap = mask(K p) by G lanes per row (G from the mean row length), partial p.Ap; the last block forms
//                   alpha (or flags a breakdown).
//   2. k_csr_update: x += alpha p, r -= alpha Ap, z = D^-1 r, partials r.z and r.r; the last block tests |r| <= tol
//                    |b| (lin3d._pcg's rule, tested every iteration) and forms beta.
//   3. k_csr_pupdate: p = z + beta p.
// Every kernel returns at once when the solve is done, so blocks of iterations can be replayed as CUDA graphs (the
// iteration number lives in device memory); the host polls the done flag between blocks.
#include <cstdint>

#include "../../include/lpm_b200.h"
#include "lpm_common.cuh"
#include "lpm_graph.h"

namespace lpm {

namespace {

constexpr int CT = 256;  // threads per block

struct CsrState {
    double rz;       // r.z of the current iteration
    double alpha, beta;
    double bn;       // |b|
    double relres;   // |r| / |b| at the last test
    int it;          // completed iterations
    int done;        // 1 once converged, broken down or out of iterations
    int status;      // LPM_STATUS_*
    int maxit;
    double tol;
    unsigned cnt[2];  // last-block counters of the two reducing kernels
};

__device__ __forceinline__ bool last_block(unsigned* cnt, bool* flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        *flag = atomicAdd(cnt, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return *flag;
}

// Sum of the per-block partials part[0..nblk) in fixed order by the last block; valid in thread 0.
__device__ __forceinline__ double sum_parts(const double* part, int nblk, double* red)
{
    double a = 0.0;
    for (int b = threadIdx.x; b < nblk; b += CT) a += __ldcg(part + b);
    return block_sum(a, red);
}

__global__ void __launch_bounds__(CT) k_csr_diag_inv(int64_t n, const int64_t* __restrict__ rp,
                                                     const int32_t* __restrict__ col, const double* __restrict__ val,
                                                     const uint8_t* __restrict__ mask, double* __restrict__ dinv,
                                                     int* bad)
{
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT) {
        double d = 0.0;
        for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
            if (col[e] == i) d += val[e];
        const bool fr = !mask || mask[i];
        if (fr && !(d > 0.0)) atomicExch(bad, 1);
        dinv[i] = fr && d > 0.0 ? 1.0 / d : 0.0;
    }
}

// r = mask(b), x = 0, z = D^-1 r, p = z; |b|^2 and r.z partials; the last block initialises the state.
__global__ void __launch_bounds__(CT) k_csr_init(int64_t n, const uint8_t* __restrict__ mask,
                                                 const double* __restrict__ b, const double* __restrict__ dinv,
                                                 double* __restrict__ x, double* __restrict__ r,
                                                 double* __restrict__ p, double* part, CsrState* S, double tol,
                                                 int maxit, const int* bad)
{
    __shared__ double red[32];
    __shared__ bool lastf;
    double bb = 0.0, rz = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT) {
        const double ri = (!mask || mask[i]) ? b[i] : 0.0;
        const double zi = dinv[i] * ri;
        x[i] = 0.0;
        r[i] = ri;
        p[i] = zi;
        bb += ri * ri;
        rz += ri * zi;
    }
    const int nb = gridDim.x;
    bb = block_sum(bb, red);
    if (threadIdx.x == 0) part[blockIdx.x] = bb;
    rz = block_sum(rz, red);
    if (threadIdx.x == 0) part[nb + blockIdx.x] = rz;
    if (!last_block(&S->cnt[0], &lastf)) return;
    const double B2 = sum_parts(part, nb, red);
    const double RZ = sum_parts(part + nb, nb, red);
    if (threadIdx.x == 0) {
        S->cnt[0] = 0u;
        S->cnt[1] = 0u;
        S->tol = tol;
        S->maxit = maxit;
        S->it = 0;
        S->bn = sqrt(B2);
        S->rz = RZ;
        S->alpha = S->beta = 0.0;
        if (*bad) {  // a free row without a positive diagonal: K_ff is not SPD
            S->relres = 1.0;
            S->status = LPM_STATUS_BREAKDOWN;
            S->done = 1;
        } else if (B2 == 0.0) {  // b = 0: x = 0 is the answer (lin3d.py:478-480)
            S->relres = 0.0;
            S->status = LPM_STATUS_OK;
            S->done = 1;
        } else {
            S->relres = 1.0;
            S->status = LPM_STATUS_NOT_CONVERGED;
            S->done = maxit <= 0 ? 1 : 0;
        }
    }
}

template <int G>
__global__ void __launch_bounds__(CT) k_csr_spmv(int64_t n, const int64_t* __restrict__ rp,
                                                 const int32_t* __restrict__ col, const double* __restrict__ val,
                                                 const uint8_t* __restrict__ mask, const double* __restrict__ p,
                                                 double* __restrict__ Ap, double* part, CsrState* S)
{
    __shared__ double red[32];
    __shared__ bool lastf;
    if (S->done) return;
    const int sub = threadIdx.x % G;
    const int64_t rows_per_pass = (int64_t)gridDim.x * (CT / G);
    double pap = 0.0;
    // the row base is uniform over the block, so every lane takes the same passes and joins every shuffle
    for (int64_t base = (int64_t)blockIdx.x * (CT / G); base < n; base += rows_per_pass) {
        const int64_t i = base + threadIdx.x / G;
        double acc = 0.0;
        if (i < n) {
            const int64_t e1 = rp[i + 1];
            for (int64_t e = rp[i] + sub; e < e1; e += G) acc += val[e] * __ldg(p + col[e]);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, G);
        if (sub == 0 && i < n) {
            const double a = (!mask || mask[i]) ? acc : 0.0;
            Ap[i] = a;
            pap += a * p[i];
        }
    }
    pap = block_sum(pap, red);
    if (threadIdx.x == 0) part[blockIdx.x] = pap;
    if (!last_block(&S->cnt[0], &lastf)) return;
    const double PAP = sum_parts(part, gridDim.x, red);
    if (threadIdx.x == 0) {
        S->cnt[0] = 0u;
        if (!(PAP > 0.0) || !isfinite(PAP)) {
            S->status = LPM_STATUS_BREAKDOWN;
            S->done = 1;
        } else {
            S->alpha = S->rz / PAP;
        }
    }
}

__global__ void __launch_bounds__(CT) k_csr_update(int64_t n, const double* __restrict__ dinv,
                                                   const double* __restrict__ p, const double* __restrict__ Ap,
                                                   double* __restrict__ x, double* __restrict__ r,
                                                   double* __restrict__ z, double* part, CsrState* S)
{
    __shared__ double red[32];
    __shared__ bool lastf;
    if (S->done) return;
    const double alpha = S->alpha;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        const double zi = dinv[i] * ri;
        z[i] = zi;
        rz += ri * zi;
        rr += ri * ri;
    }
    const int nb = gridDim.x;
    rz = block_sum(rz, red);
    if (threadIdx.x == 0) part[blockIdx.x] = rz;
    rr = block_sum(rr, red);
    if (threadIdx.x == 0) part[nb + blockIdx.x] = rr;
    if (!last_block(&S->cnt[1], &lastf)) return;
    const double RZ = sum_parts(part, nb, red);
    const double RR = sum_parts(part + nb, nb, red);
    if (threadIdx.x == 0) {
        S->cnt[1] = 0u;
        const int it = S->it + 1;
        S->it = it;
        const double rel = sqrt(RR) / S->bn;
        S->relres = rel;
        if (!isfinite(rel) || !isfinite(RZ)) {
            S->status = LPM_STATUS_BREAKDOWN;
            S->done = 1;
        } else if (rel <= S->tol) {
            S->status = LPM_STATUS_OK;
            S->done = 1;
        } else if (it >= S->maxit) {
            S->status = LPM_STATUS_NOT_CONVERGED;
            S->done = 1;
        } else {
            S->beta = RZ / S->rz;
            S->rz = RZ;
        }
    }
}

__global__ void __launch_bounds__(CT) k_csr_pupdate(int64_t n, const double* __restrict__ z, double* __restrict__ p,
                                                    const CsrState* S)
{
    if (S->done) return;
    const double beta = S->beta;
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT)
        p[i] = z[i] + beta * p[i];
}

int csr_grid(int64_t n, int rows_per_block)
{
    const int64_t need = (n + rows_per_block - 1) / rows_per_block;
    return (int)(need < 148 * 8 ? (need < 1 ? 1 : need) : 148 * 8);
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

size_t csr_workspace_bytes(int64_t n)
{
    const size_t vec = align256((size_t)n * sizeof(double));
    // r, p, z, Ap, D^-1; partials; state; error flag; alignment slack of the base pointer
    return 5 * vec + align256(2 * 148 * 8 * sizeof(double)) + align256(sizeof(CsrState)) + 256 + 256;
}

}  // namespace lpm

using namespace lpm;

int64_t lpm_csr_workspace_bytes(int64_t n)
{
    if (n < 1) return LPM_ERR_ARG;
    return (int64_t)csr_workspace_bytes(n);
}

int lpm_csr_pcg_f64(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, const uint8_t* mask,
                    const double* b, double* x, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                    int32_t* iters, double* relres, int32_t* status, void* stream)
{
    if (n < 1 || n > INT32_MAX || !rowptr || !col || !val || !b || !x || !opts || !workspace || !iters || !relres ||
        !status)
        return LPM_ERR_ARG;
    if (opts->tol < 0.0 || opts->maxit < 0) return LPM_ERR_ARG;
    if (workspace_bytes < csr_workspace_bytes(n)) return LPM_ERR_WORKSPACE;
    cudaStream_t st = (cudaStream_t)stream;
    // workspace: r, p, z, Ap, D^-1, partials, state, error flag (256-byte aligned pieces)
    unsigned char* w = reinterpret_cast<unsigned char*>(((uintptr_t)workspace + 255) & ~(uintptr_t)255);
    const size_t vec = align256((size_t)n * sizeof(double));
    double* r = reinterpret_cast<double*>(w);
    double* p = reinterpret_cast<double*>(w + vec);
    double* z = reinterpret_cast<double*>(w + 2 * vec);
    double* Ap = reinterpret_cast<double*>(w + 3 * vec);
    double* dinv = reinterpret_cast<double*>(w + 4 * vec);
    double* part = reinterpret_cast<double*>(w + 5 * vec);
    CsrState* S = reinterpret_cast<CsrState*>(w + 5 * vec + align256(2 * 148 * 8 * sizeof(double)));
    int* bad = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(S) + align256(sizeof(CsrState)));

    cudaError_t e = cudaMemsetAsync(S, 0, sizeof(CsrState), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    const int gv = csr_grid(n, CT);
    k_csr_diag_inv<<<gv, CT, 0, st>>>(n, rowptr, col, val, mask, dinv, bad);
    k_csr_init<<<gv, CT, 0, st>>>(n, mask, b, dinv, x, r, p, part, S, opts->tol, opts->maxit, bad);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    // lanes per row from the mean row length (coalesced column/value reads for lattice rows of ~18-50 entries)
    int64_t nnz = 0;
    if ((e = cudaMemcpyAsync(&nnz, rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return (int)e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return (int)e;
    const double mean = (double)nnz / (double)n;
    const int G = mean <= 6 ? 4 : mean <= 20 ? 8 : mean <= 64 ? 16 : 32;
    const int gs = csr_grid(n, CT / G);
    const int poll = opts->poll > 0 ? opts->poll : 32;
    auto one_iter = [&](int, cudaStream_t s) -> cudaError_t {
        switch (G) {
        case 4: k_csr_spmv<4><<<gs, CT, 0, s>>>(n, rowptr, col, val, mask, p, Ap, part, S); break;
        case 8: k_csr_spmv<8><<<gs, CT, 0, s>>>(n, rowptr, col, val, mask, p, Ap, part, S); break;
        case 16: k_csr_spmv<16><<<gs, CT, 0, s>>>(n, rowptr, col, val, mask, p, Ap, part, S); break;
        default: k_csr_spmv<32><<<gs, CT, 0, s>>>(n, rowptr, col, val, mask, p, Ap, part, S); break;
        }
        k_csr_update<<<gv, CT, 0, s>>>(n, dinv, p, Ap, x, r, z, part, S);
        k_csr_pupdate<<<gv, CT, 0, s>>>(n, z, p, S);
        return cudaGetLastError();
    };
    GraphKey key;
    key.ptr = {rowptr, col, val, mask, b, x, workspace, nullptr, nullptr, nullptr};
    key.val[0] = n;
    key.val[1] = G;
    key.val[2] = poll;
    key.val[3] = 0x435352;  // distinguishes this engine's graphs from the lattice engines'
    int done = 0;
    for (int it = 0;; it += poll) {
        if ((e = cudaMemcpyAsync(&done, &S->done, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return (int)e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return (int)e;
        if (done) break;
        if ((e = run_iteration_block(opts->prof == nullptr, key, it, poll, st, one_iter)) != cudaSuccess)
            return (int)e;
    }
    // outputs are device arrays of one element, as the batched engines' per-system outputs
    if ((e = cudaMemcpyAsync(iters, &S->it, sizeof(int32_t), cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(relres, &S->relres, sizeof(double), cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(status, &S->status, sizeof(int32_t), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return (int)e;
    return LPM_OK;
}
