// Batched CG / block-Jacobi PCG on the free DOFs of many LPM systems at once, and the mixed-precision driver.
//
// Algorithm per system (coarse3d/lin3d.py:464-518, with the batching / freezing rules of
// coarse3d/torch_lpm3d.py:109-140):
//   r = mask(b - K x);  z = mask(M r);  p = z;  rz = r.z;  bn = |b|
//   repeat:  Ap = mask(K p);  alpha = rz / p.Ap;  x += alpha p;  r -= alpha Ap
//            every `check` iterations (and at maxit): rel = |r| / bn; a system with rel <= tol is frozen
//            z = mask(M r);  beta = r.z_new / rz;  p = z + beta p
// Vectors are in T (float or double); inner products and scalars are FP64.  Reductions are deterministic: per-block
// partials, summed in a fixed order by the last block of each system, which also performs that system's scalar step
// (beta, convergence test, freezing).  The host loop reads one counter every `poll` iterations.
//
// Mixed precision (iterative refinement): the true residual r = mask(b - K x) is formed in FP64 with the FP64
// coefficients; each correction solves K d = r / |r| with the FP32 PCG to a loose tolerance; x += |r| d in FP64; the
// stopping test is on the FP64 true residual.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lpm_amg.h"
#include "lpm_cg.h"
#include "lpm_graph.h"
#include "lpm_tma.h"

namespace lpm {

namespace {

constexpr int VB = 256;  // vector-kernel block

template <typename T, int DIM>
__device__ __forceinline__ void block_mv(const T* __restrict__ M, const T* r, T* z)
{
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        T acc = 0;
#pragma unroll
        for (int b = 0; b < DIM; ++b) acc += M[a * DIM + b] * r[b];
        z[a] = acc;
    }
}

// Block sums of NV values at once: the arithmetic of block_sum (a shuffle tree per warp, then one over the warp
// sums) for each value, with one pair of barriers for all of them; results valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum_n(double (&v)[NV], double* sh)
{
    const int tid = threadIdx.x, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
    __syncthreads();  // sh is no longer read by an earlier reduction
    if ((tid & 31) == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) sh[j * 32 + (tid >> 5)] = v[j];
    }
    __syncthreads();
    if (tid < 32) {
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = warp_sum(tid < nw ? sh[j * 32 + tid] : 0.0);
    }
}

// Deterministic reduction of NV per-thread values per system.  Every block writes its NV block sums to
// part[(j*nsys + s)*nblk + b]; the last block of system s (one counter per system) sums the rows in fixed order.
// Returns true in that block; totals valid in thread 0.
template <int NV>
__device__ __forceinline__ bool reduce_last(const double (&v)[NV], double* part, unsigned* cnt, int s, int nsys,
                                            int b, int nblk, double (&tot)[NV])
{
    __shared__ bool is_last;
    __shared__ double shn[NV * 32];
    const int tid = threadIdx.x;
    double bs[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) bs[j] = v[j];
    block_sum_n<NV>(bs, shn);
    if (tid == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) part[((int64_t)j * nsys + s) * nblk + b] = bs[j];
        __threadfence();
        is_last = atomicAdd(cnt + s, 1u) == (unsigned)(nblk - 1);
    }
    __syncthreads();
    if (!is_last) return false;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double acc = 0.0;
        const double* row = part + ((int64_t)j * nsys + s) * nblk;
        for (int k = tid; k < nblk; k += blockDim.x) acc += __ldcg(row + k);
        tot[j] = acc;
    }
    block_sum_n<NV>(tot, shn);
    if (tid == 0) cnt[s] = 0u;
    return true;
}

// ------------------------------------------------------------------------------------------------------- init
template <typename T, int DIM, bool PREC>
__global__ void __launch_bounds__(VB) k_cg_init(int64_t N, int sys0, Batch bt, const T* __restrict__ b,
                                                const T* __restrict__ Ax, const uint8_t* __restrict__ mask,
                                                const T* __restrict__ Minv, T* __restrict__ r, T* __restrict__ z,
                                                T* __restrict__ p, CgScalars sc, double tol, int precheck)
{
    const int s = sys0 + blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};  // b.b, r.z, r.r
    if (i < N) {
        const int64_t o = ((int64_t)s * N + i) * DIM;
        const uint8_t* m = mask ? mask + ((int64_t)(s % bt.nmask) * N + i) * DIM : nullptr;
        T rv[DIM], zv[DIM];
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            const T bv = b[o + a];
            T w = Ax ? bv - Ax[o + a] : bv;
            if (m && !m[a]) w = T(0);
            rv[a] = w;
            v[0] += (double)bv * (double)bv;
        }
        if constexpr (PREC) {
            block_mv<T, DIM>(Minv + ((int64_t)(s / bt.rhs_per_set) * N + i) * DIM * DIM, rv, zv);
#pragma unroll
            for (int a = 0; a < DIM; ++a)
                if (m && !m[a]) zv[a] = T(0);
        } else {
#pragma unroll
            for (int a = 0; a < DIM; ++a) zv[a] = rv[a];
        }
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            r[o + a] = rv[a];
            if constexpr (PREC) z[o + a] = zv[a];
            p[o + a] = zv[a];
            v[1] += (double)rv[a] * (double)zv[a];
            v[2] += (double)rv[a] * (double)rv[a];
        }
    }
    double tot[3];
    if (!reduce_last<3>(v, sc.part, sc.cnt, s, bt.nsys, blockIdx.x, gridDim.x, tot) || threadIdx.x != 0) return;
    const double bn = sqrt(tot[0]);
    const double rel = bn > 0.0 ? sqrt(tot[2]) / bn : 0.0;
    const bool finite = isfinite(bn) && isfinite(tot[1]) && isfinite(tot[2]);
    int act = bn > 0.0 && finite;
    if (act && precheck && rel <= (sc.tols ? sc.tols[s] : tol)) act = 0;
    sc.bn[s] = bn;
    sc.rz[s] = tot[1];
    sc.rr[s] = tot[2];
    sc.beta[s] = 0.0;  // the fused p-update's first p' = z + 0 p
    sc.act[s] = act;
    sc.iters[s] = 0;
    sc.relres[s] = rel;
    sc.status[s] = finite ? LPM_STATUS_OK : LPM_STATUS_BREAKDOWN;
    if (!act) atomicAdd(sc.nconv, 1u);
}

// ----------------------------------------------------------------------------------------------------- update
// PF (fused p-update, full 2D boxes): the operator formed p' = z + beta p into one of the buffers p / p1 by the
// parity of pk[s], the system's count of completed iterations; this kernel reads p' from there, takes its iteration
// number from pk[s], and its last block advances pk[s] (every block of the system has read it by then).
template <typename T, int DIM, bool PREC, bool PF = false>
__global__ void __launch_bounds__(VB) k_cg_update(int64_t N, int sys0, Batch bt, int it_host, int check,
                                                  int maxit, double tol, const uint8_t* __restrict__ mask,
                                                  const T* __restrict__ Minv, T* __restrict__ x, T* __restrict__ r,
                                                  T* __restrict__ z, const T* __restrict__ p0,
                                                  const T* __restrict__ Ap, CgScalars sc,
                                                  const T* __restrict__ p1 = nullptr, int* __restrict__ pk = nullptr)
{
    const int s = sys0 + blockIdx.y;
    // a frozen system: every block of it leaves before the reduction, so its counter stays at zero
    if (!sc.act[s]) return;
    const int it = PF ? pk[s] + 1 : (sc.itp ? *sc.itp : it_host);
    const T* __restrict__ p = PF && (pk[s] & 1) == 0 ? p1 : p0;
    const int cur = (it - 1) & 1, nxt = it & 1;
    const double pAp = sc.pAp[s];
    const double rzc = sc.rz[cur * bt.nsys + s];
    const bool good = pAp > 0.0 && isfinite(pAp) && isfinite(rzc);
    const double alpha = good ? rzc / pAp : 0.0;
    double v[2] = {0.0, 0.0};  // r.z, r.r
    // grid-stride over particles: a few blocks per system, so the reduction epilogue is amortised
    for (int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x; i < N; i += (int64_t)gridDim.x * VB) {
        const int64_t o = ((int64_t)s * N + i) * DIM;
        const T al = (T)alpha;
        T rv[DIM], zv[DIM];
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            x[o + a] += al * p[o + a];
            rv[a] = r[o + a] - al * Ap[o + a];
            r[o + a] = rv[a];
        }
        if constexpr (PREC) {
            const uint8_t* m = mask ? mask + ((int64_t)(s % bt.nmask) * N + i) * DIM : nullptr;
            block_mv<T, DIM>(Minv + ((int64_t)(s / bt.rhs_per_set) * N + i) * DIM * DIM, rv, zv);
#pragma unroll
            for (int a = 0; a < DIM; ++a) {
                if (m && !m[a]) zv[a] = T(0);
                z[o + a] = zv[a];
            }
        } else {
#pragma unroll
            for (int a = 0; a < DIM; ++a) zv[a] = rv[a];
        }
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            v[0] += (double)rv[a] * (double)zv[a];
            v[1] += (double)rv[a] * (double)rv[a];
        }
    }
    double tot[2];
    if (!reduce_last<2>(v, sc.part, sc.cnt, s, bt.nsys, blockIdx.x, gridDim.x, tot) || threadIdx.x != 0) return;
    if constexpr (PF) pk[s] = it;
    const double rzn = tot[0], rrn = tot[1];
    sc.rz[nxt * bt.nsys + s] = rzn;
    sc.rr[s] = rrn;
    sc.beta[s] = rzc != 0.0 ? rzn / rzc : 0.0;
    const double rel = sqrt(rrn) / sc.bn[s];
    const double tl = sc.tols ? sc.tols[s] : tol;
    if (!isfinite(pAp) || pAp < 0.0 || !isfinite(rrn) || !isfinite(rzn)) {
        sc.act[s] = 0;
        sc.iters[s] = it;
        sc.relres[s] = rel;
        sc.status[s] = LPM_STATUS_BREAKDOWN;
        atomicAdd(sc.nconv, 1u);
        return;
    }
    if (it % check == 0 || it == maxit) {
        sc.relres[s] = rel;
        if (rel <= tl || it == maxit) {
            sc.act[s] = 0;
            sc.iters[s] = it;
            if (rel > tl) sc.status[s] = LPM_STATUS_NOT_CONVERGED;
            atomicAdd(sc.nconv, 1u);
        }
    }
}

// p = z + beta p   (plain CG: z == r)
template <typename T, int DIM>
__global__ void __launch_bounds__(VB) k_cg_pupdate(int64_t N, int sys0, const T* __restrict__ z, T* __restrict__ p,
                                                   CgScalars sc)
{
    if (sc.itp && sys0 == 0 && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(sc.itp, 1);
    const int s = sys0 + blockIdx.y;
    if (!sc.act[s]) return;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    const T be = (T)sc.beta[s];
    const int64_t o = ((int64_t)s * N + i) * DIM;
#pragma unroll
    for (int a = 0; a < DIM; ++a) p[o + a] = z[o + a] + be * p[o + a];
}

// ------------------------------------------------------------------------------------------- refinement kernels
// r64 = mask(b - Kx) (Kx may be null: x == 0); per-system |r|^2 -> rn2, |b|^2 -> bn2.
template <int DIM>
__global__ void __launch_bounds__(VB) k_ir_residual(int64_t N, int sys0, Batch bt, const double* __restrict__ b,
                                                    const double* __restrict__ Kx,
                                                    const uint8_t* __restrict__ mask, double* __restrict__ r,
                                                    double* part, unsigned* cnt, double* rn2, double* bn2)
{
    const int s = sys0 + blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < N) {
        const int64_t o = ((int64_t)s * N + i) * DIM;
        const uint8_t* m = mask ? mask + ((int64_t)(s % bt.nmask) * N + i) * DIM : nullptr;
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            const double bv = b[o + a];
            double w = Kx ? bv - Kx[o + a] : bv;
            if (m && !m[a]) w = 0.0;
            r[o + a] = w;
            v[0] += w * w;
            v[1] += bv * bv;
        }
    }
    double tot[2];
    if (reduce_last<2>(v, part, cnt, s, bt.nsys, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        rn2[s] = tot[0];
        bn2[s] = tot[1];
    }
}

// r32 = r64 * scale[s] (1/|r| for active systems, 0 otherwise); d32 = 0
template <int DIM>
__global__ void __launch_bounds__(VB) k_ir_scale(int64_t N, int sys0, const double* __restrict__ r64,
                                                 const double* __restrict__ scale, float* __restrict__ r32,
                                                 float* __restrict__ d32)
{
    const int s = sys0 + blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    const double sc = scale[s];
    const int64_t o = ((int64_t)s * N + i) * DIM;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        r32[o + a] = (float)(r64[o + a] * sc);
        d32[o + a] = 0.0f;
    }
}

// x64 += step[s] * d32
template <int DIM>
__global__ void __launch_bounds__(VB) k_ir_correct(int64_t N, int sys0, const double* __restrict__ step,
                                                   const float* __restrict__ d32, double* __restrict__ x)
{
    const int s = sys0 + blockIdx.y;
    const double st = step[s];
    if (st == 0.0) return;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    const int64_t o = ((int64_t)s * N + i) * DIM;
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[o + a] += st * (double)d32[o + a];
}

// ---------------------------------------------------------------------------------------------- workspace
inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

struct Carver {
    char* base;
    size_t off;
    template <typename X>
    X* take(size_t count)
    {
        X* p = base ? reinterpret_cast<X*>(base + off) : nullptr;
        off = align_up(off + count * sizeof(X));
        return p;
    }
};

inline int vec_blocks(int64_t N) { return (int)((N + VB - 1) / VB); }

template <typename T>
struct CgWork {
    T *r, *z, *p, *Ap, *st;
    CgScalars sc;
    double* mv_part;
    double* mv_final;
    unsigned* mv_cnt;
    int* pk;  // completed iterations per system (the fused p-update's buffer parity)
};

// The fused p-update runs where the operator is a 2D tile kernel (k_sq_fused, k_sq_multi): full 2D boxes.  Its
// second p buffer is the shell-sum scratch `st`, which the 2D tile operators do not use.
inline bool pfused(const Lattice& L) { return L.dim == 2 && L.nbr == nullptr; }

template <typename T>
void carve_cg(Carver& cv, const Lattice& L, int nsys, bool precond, CgWork<T>& w)
{
    const size_t nv = (size_t)nsys * L.N * L.dim;
    const int nb = vec_blocks(L.N);
    w.r = cv.take<T>(nv);
    w.z = precond ? cv.take<T>(nv) : nullptr;
    w.p = cv.take<T>(nv);
    w.Ap = cv.take<T>(nv);
    w.st = cv.take<T>((size_t)nsys * L.N * 4);
    w.sc.part = cv.take<double>((size_t)3 * nsys * nb);
    w.sc.cnt = cv.take<unsigned>(nsys);
    w.sc.bn = cv.take<double>(nsys);
    w.sc.rz = cv.take<double>(2 * (size_t)nsys);
    w.sc.rr = cv.take<double>(nsys);
    w.sc.pAp = cv.take<double>(nsys);
    w.sc.beta = cv.take<double>(nsys);
    w.sc.act = cv.take<int>(nsys);
    w.sc.nconv = cv.take<unsigned>(1);
    w.sc.nblk = nb;
    w.mv_part = cv.take<double>((size_t)nsys * kmv_dot_blocks(L));
    w.mv_cnt = cv.take<unsigned>(nsys);
    w.mv_final = w.sc.pAp;
    w.sc.itp = cv.take<int>(1);
    w.pk = cv.take<int>(nsys);
}

template <typename T>
struct IrWork {
    double *r64, *Kx, *st64, *scal;  // scal: rn2, bn2, scale, step (4*nsys)
    double* part;
    unsigned* cnt;
    float *r32, *d32;
    int *it_in, *st_in;
    double *rel_in, *itol;
    void* cg_ws;
    size_t cg_bytes;
};

void carve_ir(Carver& cv, const Lattice& L, const Batch& bt, bool precond, IrWork<float>& w)
{
    const int nsys = bt.nsys;
    const size_t nv = (size_t)nsys * L.N * L.dim;
    w.r64 = cv.take<double>(nv);
    w.Kx = cv.take<double>(nv);
    w.st64 = cv.take<double>((size_t)nsys * L.N * 4);
    w.scal = cv.take<double>(4 * (size_t)nsys);
    w.part = cv.take<double>((size_t)2 * nsys * vec_blocks(L.N));
    w.cnt = cv.take<unsigned>(nsys);
    w.r32 = cv.take<float>(nv);
    w.d32 = cv.take<float>(nv);
    w.it_in = cv.take<int>(nsys);
    w.st_in = cv.take<int>(nsys);
    w.rel_in = cv.take<double>(nsys);
    w.itol = cv.take<double>(nsys);
    w.cg_bytes = cg_workspace_bytes(L, bt, LPM_F32, precond);
    w.cg_ws = cv.take<char>(w.cg_bytes);
}

// Blocks per system of the update kernel: about eight resident blocks per SM over the whole launch, at most one
// per 256 particles.
inline int update_blocks(int nb, int ns)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ||
            sms < 1)
            sms = 148;
    }
    return std::max(1, std::min(nb, (8 * sms + ns - 1) / ns));
}

template <typename T, int DIM>
void launch_update(dim3 g, cudaStream_t st, bool precond, const Batch& bt, int64_t N, int s0, int it,
                   const lpm_cg_opts& o, const uint8_t* mask, const T* Minv, T* x, CgWork<T>& w, bool pf = false)
{
    const dim3 gu(update_blocks((int)g.x, (int)g.y), g.y);
    if (pf) {  // p' comes from the operator: no p-update kernel
        if (precond)
            k_cg_update<T, DIM, true, true><<<gu, VB, 0, st>>>(N, s0, bt, it, o.check, o.maxit, o.tol, mask, Minv,
                                                               x, w.r, w.z, w.p, w.Ap, w.sc, w.st, w.pk);
        else
            k_cg_update<T, DIM, false, true><<<gu, VB, 0, st>>>(N, s0, bt, it, o.check, o.maxit, o.tol, mask, Minv,
                                                                x, w.r, w.z, w.p, w.Ap, w.sc, w.st, w.pk);
        return;
    }
    if (precond)
        k_cg_update<T, DIM, true><<<gu, VB, 0, st>>>(N, s0, bt, it, o.check, o.maxit, o.tol, mask, Minv, x, w.r,
                                                     w.z, w.p, w.Ap, w.sc);
    else
        k_cg_update<T, DIM, false><<<gu, VB, 0, st>>>(N, s0, bt, it, o.check, o.maxit, o.tol, mask, Minv, x, w.r,
                                                      w.z, w.p, w.Ap, w.sc);
    k_cg_pupdate<T, DIM><<<g, VB, 0, st>>>(N, s0, precond ? w.z : w.r, w.p, w.sc);
}

template <typename T, int DIM>
void launch_init(dim3 g, cudaStream_t st, bool precond, const Batch& bt, int64_t N, int s0, const T* b, const T* Ax,
                 const uint8_t* mask, const T* Minv, CgWork<T>& w, const lpm_cg_opts& o)
{
    if (precond)
        k_cg_init<T, DIM, true><<<g, VB, 0, st>>>(N, s0, bt, b, Ax, mask, Minv, w.r, w.z, w.p, w.sc, o.tol,
                                                  o.precheck);
    else
        k_cg_init<T, DIM, false><<<g, VB, 0, st>>>(N, s0, bt, b, Ax, mask, Minv, w.r, w.z, w.p, w.sc, o.tol,
                                                   o.precheck);
}

}  // namespace

static bool fused_ok(const Lattice& L, const CoefLayout& cl, int elem_bytes)
{
    return L.dim == 3 && L.nbr == nullptr && cl.slot_stride == L.N && cl.site_stride == 1 &&
           tma_supported(L.nx, elem_bytes);
}

size_t cg_workspace_bytes(const Lattice& L, const Batch& bt, int precision, int precond)
{
    Carver cv{nullptr, 0};
    if (precision == LPM_F32) {
        CgWork<float> w;
        carve_cg<float>(cv, L, bt.nsys, precond != 0, w);
    } else {
        CgWork<double> w;
        carve_cg<double>(cv, L, bt.nsys, precond != 0, w);
    }
    size_t n = cv.off + 256;
    const int es = precision == LPM_F32 ? 4 : 8;
    if (L.dim == 3 && L.nbr == nullptr && tma_supported(L.nx, es))
        n = std::max(n, cg_fused_workspace_bytes(L, bt.nsys, bt.rhs_per_set, es, precond));
    if (persist_fits(L, bt)) n = std::max(n, persist_workspace_bytes(L, bt, es));
    return n;
}

size_t ir_workspace_bytes(const Lattice& L, const Batch& bt, int precond)
{
    Carver cv{nullptr, 0};
    IrWork<float> w;
    carve_ir(cv, L, bt, precond != 0, w);
    return cv.off + 256;
}

template <typename T>
int cg_solve(const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt, const T* Minv,
             const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws, size_t ws_bytes,
             int* iters, double* relres, int* status, cudaStream_t st)
{
    if (o.maxit < 0 || o.check < 1 || o.poll < 1 || bt.nsys < 1) return LPM_ERR_ARG;
    if (o.engine < LPM_ENGINE_AUTO || o.engine > LPM_ENGINE_PERSISTENT) return LPM_ERR_ARG;
    if (o.engine == LPM_ENGINE_PERSISTENT || (o.engine == LPM_ENGINE_AUTO && !o.prof && persist_auto(L, bt, (int)sizeof(T))))
        return cg_solve_persist<T>(L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws, ws_bytes, iters, relres,
                                   status, st);
    if (fused_ok(L, cl, (int)sizeof(T)) && tma_aligned(Kn, Tv, b))
        return cg_solve_fused<T>(L, Kn, Tv, bt, Minv, mask, b, x, x_is_zero, o, ws, ws_bytes, iters, relres, status,
                                 st);
    const bool precond = Minv != nullptr;
    // align the caller's buffer
    char* base = static_cast<char*>(ws);
    const size_t shift = (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    Carver cv{base + shift, 0};
    CgWork<T> w;
    carve_cg<T>(cv, L, bt.nsys, precond, w);
    if (cv.off + shift > ws_bytes) return LPM_ERR_WORKSPACE;
    w.sc.iters = iters;
    w.sc.relres = relres;
    w.sc.status = status;
    w.sc.tols = o.tol_sys;
    const int64_t N = L.N;
    cudaError_t e = cudaMemsetAsync(w.sc.cnt, 0, sizeof(unsigned) * bt.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mv_cnt, 0, sizeof(unsigned) * bt.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.sc.nconv, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.pk, 0, sizeof(int) * bt.nsys, st);
    if (e != cudaSuccess) return (int)e;
    if (!x_is_zero) {
        e = launch_kmv<T>(L, x, Kn, Tv, cl, bt, w.Ap, w.st, nullptr, st);
        if (e != cudaSuccess) return (int)e;
    }
    const int nb = vec_blocks(N);
    for (int s0 = 0; s0 < bt.nsys; s0 += 65535) {
        const int ns = bt.nsys - s0 < 65535 ? bt.nsys - s0 : 65535;
        const dim3 g(nb, ns);
        const T* Ax = x_is_zero ? nullptr : w.Ap;
        if (L.dim == 3)
            launch_init<T, 3>(g, st, precond, bt, N, s0, b, Ax, mask, Minv, w, o);
        else
            launch_init<T, 2>(g, st, precond, bt, N, s0, b, Ax, mask, Minv, w, o);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;

    MvEpilogue ep{mask, w.mv_part, w.mv_final, w.mv_cnt, w.sc.act};
    const bool pf = pfused(L);
    if (pf) {
        ep.pz = precond ? w.z : w.r;
        ep.p0 = w.p;
        ep.p1 = w.st;
        ep.beta = w.sc.beta;
        ep.pk = w.pk;
    }
    KmvTimer timer(o.prof, st);
    unsigned nconv = 0;
    e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    static const int kOne = 1;
    if ((e = cudaMemcpyAsync(w.sc.itp, &kOne, sizeof(int), cudaMemcpyHostToDevice, st)) != cudaSuccess) return (int)e;
    auto one_iter = [&](int it, cudaStream_t s) -> cudaError_t {
        timer.begin(nconv == 0);
        cudaError_t ee = launch_kmv<T>(L, w.p, Kn, Tv, cl, bt, w.Ap, w.st, &ep, s);
        timer.end();
        if (ee != cudaSuccess) return ee;
        for (int s0 = 0; s0 < bt.nsys; s0 += 65535) {
            const int ns = bt.nsys - s0 < 65535 ? bt.nsys - s0 : 65535;
            const dim3 g(nb, ns);
            if (L.dim == 3)
                launch_update<T, 3>(g, s, precond, bt, N, s0, it, o, mask, Minv, x, w);
            else
                launch_update<T, 2>(g, s, precond, bt, N, s0, it, o, mask, Minv, x, w, pf);
        }
        return cudaGetLastError();
    };
    GraphKey key;
    key.ptr = {ws, Kn, Tv, mask, x, Minv, L.nbr, o.tol_sys, nullptr, nullptr};
    key.val = {2, bt.nsys, bt.rhs_per_set, bt.nmask, L.nx, L.ny, L.nz, o.poll, o.check, o.maxit, precond ? 1 : 0,
               (long long)sizeof(T), cl.set_stride, cl.slot_stride * 1000003LL + cl.site_stride, L.dim, 0};
    double tolv = o.tol;
    std::memcpy(&key.val[15], &tolv, sizeof(double));
    int it = 1;
    while (it <= o.maxit && nconv < (unsigned)bt.nsys) {
        const int block = std::min(o.poll - (it - 1) % o.poll, o.maxit - it + 1);
        const bool use_graph = !o.prof && it > 1 && block == o.poll;
        if ((e = run_iteration_block(use_graph, key, it, block, st, one_iter)) != cudaSuccess) return (int)e;
        it += block;
        e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return (int)e;
        timer.collect();
    }
    timer.collect();
    return LPM_OK;
}

template int cg_solve<float>(const Lattice&, const float*, const float*, const CoefLayout&, const Batch&,
                             const float*, const uint8_t*, const float*, float*, int, const lpm_cg_opts&, void*,
                             size_t, int*, double*, int*, cudaStream_t);
template int cg_solve<double>(const Lattice&, const double*, const double*, const CoefLayout&, const Batch&,
                              const double*, const uint8_t*, const double*, double*, int, const lpm_cg_opts&, void*,
                              size_t, int*, double*, int*, cudaStream_t);

int ir_solve(const Lattice& L, const double* Kn64, const double* Tv64, const CoefLayout& cl64, const float* Kn32,
             const float* Tv32, const CoefLayout& cl32, const float* Minv32, const Batch& bt, const uint8_t* mask,
             const double* b, double* x, const lpm_ir_opts& o, void* ws, size_t ws_bytes, int* iters,
             double* relres, int* status, int* outer, cudaStream_t st, lpm_amg* amg)
{
    if (o.maxit < 1 || o.max_outer < 1 || o.check < 1 || o.poll < 1 || bt.nsys < 1) return LPM_ERR_ARG;
    char* base = static_cast<char*>(ws);
    const size_t shift = (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    Carver cv{base + shift, 0};
    IrWork<float> w;
    carve_ir(cv, L, bt, Minv32 != nullptr, w);
    if (cv.off + shift > ws_bytes) return LPM_ERR_WORKSPACE;
    const int ns = bt.nsys;
    const int64_t N = L.N;
    double *rn2 = w.scal, *bn2 = w.scal + ns, *scale = w.scal + 2 * ns, *step = w.scal + 3 * ns;
    std::vector<double> h(2 * (size_t)ns), hs(2 * (size_t)ns);
    std::vector<int> h_it(ns), h_st(ns), tot_it(ns, 0), fin_st(ns, LPM_STATUS_OK);
    std::vector<double> h_rel(ns, 0.0), h_tol(ns, o.inner_tol);
    cudaError_t e = cudaMemsetAsync(w.cnt, 0, sizeof(unsigned) * ns, st);
    if (e != cudaSuccess) return (int)e;
    const int nb = vec_blocks(N);
    int steps = 0, rc = LPM_OK;
    bool x_zero = o.x_is_zero != 0;
    for (int k = 0;; ++k) {
        // true residual in FP64
        if (!x_zero) {
            if (fused_ok(L, cl64, 8) && pair64_supported(L.nx) && tma_aligned(x, Kn64, Tv64)) {
                // packed FP64 coefficients: the FP64 instantiation of the pair operator
                const PairArgs a = pair64_args(L.nx, L.ny, L.nz, N, bt.nsys, bt.rhs_per_set, x, Kn64, Tv64, w.Kx);
                e = launch_sc_pair64(a, false, st);
            } else if (fused_ok(L, cl64, 8) && tma_aligned(x, Kn64, Tv64)) {  // packed FP64 coefficients: TMA operator
                TmaArgs<double> a{};
                a.nx = L.nx;
                a.ny = L.ny;
                a.nz = L.nz;
                a.N = N;
                a.nsys = bt.nsys;
                a.rhs_per_set = bt.rhs_per_set;
                a.nmask = bt.nmask;
                tma_configure(a);
                a.u = x;
                a.Kn = Kn64;
                a.Tv = Tv64;
                a.out = w.Kx;
                e = launch_sc_tma<double>(a, false, st);
            } else {
                e = launch_kmv<double>(L, x, Kn64, Tv64, cl64, bt, w.Kx, w.st64, nullptr, st);
            }
            if (e != cudaSuccess) return (int)e;
        }
        for (int s0 = 0; s0 < ns; s0 += 65535) {
            const int nss = ns - s0 < 65535 ? ns - s0 : 65535;
            const dim3 g(nb, nss);
            if (L.dim == 3)
                k_ir_residual<3><<<g, VB, 0, st>>>(N, s0, bt, b, x_zero ? nullptr : w.Kx, mask, w.r64, w.part,
                                                   w.cnt, rn2, bn2);
            else
                k_ir_residual<2><<<g, VB, 0, st>>>(N, s0, bt, b, x_zero ? nullptr : w.Kx, mask, w.r64, w.part,
                                                   w.cnt, rn2, bn2);
        }
        e = cudaMemcpyAsync(h.data(), w.scal, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return (int)e;
        int nact = 0;
        for (int s = 0; s < ns; ++s) {
            const double rn = std::sqrt(h[s]), bn = std::sqrt(h[ns + s]);
            h_rel[s] = bn > 0 ? rn / bn : 0.0;
            const bool more = bn > 0 && std::isfinite(rn) && h_rel[s] > o.tol && tot_it[s] < o.maxit &&
                              fin_st[s] != LPM_STATUS_BREAKDOWN;
            hs[s] = more ? 1.0 / rn : 0.0;
            hs[ns + s] = more ? rn : 0.0;
            nact += more;
            if (!std::isfinite(rn)) fin_st[s] = LPM_STATUS_BREAKDOWN;
        }
        if (nact == 0 || k >= o.max_outer) break;
        ++steps;
        e = cudaMemcpyAsync(scale, hs.data(), sizeof(double) * 2 * ns, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return (int)e;
        for (int s0 = 0; s0 < ns; s0 += 65535) {
            const int nss = ns - s0 < 65535 ? ns - s0 : 65535;
            const dim3 g(nb, nss);
            if (L.dim == 3)
                k_ir_scale<3><<<g, VB, 0, st>>>(N, s0, w.r64, scale, w.r32, w.d32);
            else
                k_ir_scale<2><<<g, VB, 0, st>>>(N, s0, w.r64, scale, w.r32, w.d32);
        }
        int remaining = 0;
        for (int s = 0; s < ns; ++s) {
            remaining = std::max(remaining, o.maxit - tot_it[s]);
            // inexact refinement: an inner solve need not reduce its residual below what is left to reach tol
            // (factor 4 of margin: the FP32 operator's own error stays well inside), and never below inner_tol
            h_tol[s] = h_rel[s] > 0.0 ? std::min(0.5, std::max(o.inner_tol, 0.25 * o.tol / h_rel[s])) : o.inner_tol;
        }
        e = cudaMemcpyAsync(w.itol, h_tol.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return (int)e;
        lpm_cg_opts io{o.inner_tol, remaining, o.check, o.poll, 0, o.prof, w.itol, o.engine, 0};
        rc = amg ? amg_pcg(amg, w.r32, w.d32, io, w.it_in, w.rel_in, w.st_in, st)
                 : cg_solve<float>(L, Kn32, Tv32, cl32, bt, Minv32, mask, w.r32, w.d32, 1, io, w.cg_ws, w.cg_bytes,
                                   w.it_in, w.rel_in, w.st_in, st);
        if (rc != LPM_OK) return rc;
        e = cudaMemcpyAsync(h_it.data(), w.it_in, sizeof(int) * ns, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_st.data(), w.st_in, sizeof(int) * ns, cudaMemcpyDeviceToHost, st);
        for (int s0 = 0; s0 < ns && e == cudaSuccess; s0 += 65535) {
            const int nss = ns - s0 < 65535 ? ns - s0 : 65535;
            const dim3 g(nb, nss);
            if (L.dim == 3)
                k_ir_correct<3><<<g, VB, 0, st>>>(N, s0, step, w.d32, x);
            else
                k_ir_correct<2><<<g, VB, 0, st>>>(N, s0, step, w.d32, x);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return (int)e;
        for (int s = 0; s < ns; ++s) {
            if (hs[ns + s] == 0.0) continue;
            tot_it[s] += h_it[s];
            if (h_st[s] == LPM_STATUS_BREAKDOWN && h_it[s] <= 1) fin_st[s] = LPM_STATUS_BREAKDOWN;
        }
        x_zero = false;
    }
    for (int s = 0; s < ns; ++s)
        if (fin_st[s] == LPM_STATUS_OK && h_rel[s] > o.tol) fin_st[s] = LPM_STATUS_NOT_CONVERGED;
    e = cudaMemcpyAsync(iters, tot_it.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(relres, h_rel.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, fin_st.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    if (outer) *outer = steps;
    return LPM_OK;
}

}  // namespace lpm
