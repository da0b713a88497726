// Batched (P)CG on the TMA-fed SC operator: three kernels per iteration.
//
//   operator:  Ap = mask(K p); per-system p.Ap; its last block per system forms alpha = rz / p.Ap
//   update:    r -= alpha Ap;  z = mask(M r);  r.z, r.r per system; the last block of a system group forms beta,
//              tests convergence every `check` iterations and freezes converged systems
//   p-update:  x += alpha p;  p = mask(M r) + beta p   (z is recomputed from r instead of being stored)
// A thread of the vector kernels handles one particle for a group of up to 16 systems of one coefficient set, so
// the 3x3 preconditioner block is read once per particle and group (Minv repacked to (nset, 9, N)).  x, r and b are
// (nsys, N, 3).  In FP32 the operator is the pair-packed kernel (kmv_pair.cu) and p, Ap live in its pair layout
// (npair, N, 3, 2); its output is unmasked, so the update masks Ap (p stays zero on fixed DOFs, so p.Ap needs no
// mask).  Reductions are deterministic (per-block partials summed in fixed order by a last block).
#include <algorithm>

#include "lpm_tma.h"

namespace lpm {

namespace {

constexpr int VB = 256;
constexpr int GRP = 16;  // systems per block in the vector kernels

template <typename T>
__global__ void k_repack_M(const T* __restrict__ M, T* __restrict__ Ms, int64_t N)
{
    const int c = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
#pragma unroll
    for (int e = 0; e < 9; ++e) Ms[((int64_t)c * 9 + e) * N + i] = M[((int64_t)c * N + i) * 9 + e];
}

struct VecGeom {
    int64_t N;
    int nsys, rps, nmask;
    int ngrp;  // system groups per set = ceil(rps / GRP)
    int npp;   // pairs per set (pair layout of p and Ap)
};

// Index of component a of particle i of system s in p / Ap: (nsys, N, 3), or the pair layout (npair, N, 3, 2).
template <bool PAIRED>
__device__ __forceinline__ int64_t vix(const VecGeom& G, int s, int64_t i, int a)
{
    if constexpr (!PAIRED) {
        return ((int64_t)s * G.N + i) * 3 + a;
    } else {
        const int set = s / G.rps, j = s - set * G.rps;
        const int64_t pr = (int64_t)set * G.npp + (j >> 1);
        return ((pr * G.N + i) * 3 + a) * 2 + (j & 1);
    }
}


struct Group {
    int gid, set, s0, nsg;
};

__device__ __forceinline__ Group group_of(const VecGeom& G)
{
    Group g;
    g.gid = blockIdx.y;
    g.set = g.gid / G.ngrp;
    g.s0 = g.set * G.rps + (g.gid % G.ngrp) * GRP;
    g.nsg = min(GRP, min(G.rps - (g.gid % G.ngrp) * GRP, G.nsys - g.s0));
    return g;
}

// Warp-shuffle reduction of NV values per system, one barrier, per-block partials part[(v*nsys + s)*nblk + b];
// returns true in the last block of this system group (one counter per group).
template <int NV>
__device__ __forceinline__ bool group_reduce(double (*vals)[NV], int nsg, int s0, int nsys, double* part,
                                             unsigned* cnt, int gid, double* sh, bool* last)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < GRP; ++j) {
        if (j >= nsg) break;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double t = warp_sum(vals[j][v]);
            if (lane == 0) sh[(j * NV + v) * 8 + w] = t;
        }
    }
    __syncthreads();
    const int nblk = gridDim.x;
    for (int t = threadIdx.x; t < nsg * NV; t += blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < nw; ++q) acc += sh[t * 8 + q];
        const int j = t / NV, v = t % NV;
        part[((int64_t)v * nsys + s0 + j) * nblk + blockIdx.x] = acc;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *last = atomicAdd(cnt + gid, 1u) == (unsigned)(nblk - 1);
    __syncthreads();
    return *last;
}

// Fixed-order total of part row (v, s) by one warp; valid in lane 0.
__device__ __forceinline__ double row_total(const double* part, int v, int s, int nsys, int nblk)
{
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int b = lane; b < nblk; b += 32) acc += __ldcg(part + ((int64_t)v * nsys + s) * nblk + b);
    return warp_sum(acc);
}

template <typename T, bool PREC>
__device__ __forceinline__ void precond(const T* m9, const uint8_t* m, const T* rv, T* zv)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        zv[a] = PREC ? m9[3 * a] * rv[0] + m9[3 * a + 1] * rv[1] + m9[3 * a + 2] * rv[2] : rv[a];
        if (m && !m[a]) zv[a] = T(0);
    }
}

// ------------------------------------------------------------------------------------------------------- init
template <typename T, bool PREC, bool PAIRED>
__global__ void __launch_bounds__(VB) k_fcg_init(VecGeom G, const T* __restrict__ b, const T* __restrict__ Ax,
                                                 const uint8_t* __restrict__ mask, const T* __restrict__ Ms,
                                                 T* __restrict__ r, T* __restrict__ p, FcgScalars sc, double* part,
                                                 unsigned* cnt, double tol, int precheck)
{
    __shared__ double sh[GRP * 3 * 8];
    __shared__ bool last;
    const Group gr = group_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    double vals[GRP][3];
    T m9[9];
    if (PREC && i < N) {
#pragma unroll
        for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)gr.set * 9 + e) * N + i];
    }
#pragma unroll
    for (int j = 0; j < GRP; ++j) {
        vals[j][0] = vals[j][1] = vals[j][2] = 0.0;
        if (j >= gr.nsg || i >= N) continue;
        const int s = gr.s0 + j;
        const int64_t o = ((int64_t)s * N + i) * 3;
        const uint8_t* m = mask ? mask + ((int64_t)(s % G.nmask) * N + i) * 3 : nullptr;
        T rv[3], zv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T bv = b[o + a];
            T w = Ax ? bv - Ax[vix<PAIRED>(G, s, i, a)] : bv;
            if (m && !m[a]) w = T(0);
            rv[a] = w;
            vals[j][0] += (double)bv * (double)bv;
        }
        precond<T, PREC>(m9, m, rv, zv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            r[o + a] = rv[a];
            p[vix<PAIRED>(G, s, i, a)] = zv[a];
            vals[j][1] += (double)rv[a] * (double)zv[a];
            vals[j][2] += (double)rv[a] * (double)rv[a];
        }
    }
    if (!group_reduce<3>(vals, gr.nsg, gr.s0, G.nsys, part, cnt, gr.gid, sh, &last)) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = w; j < gr.nsg; j += VB / 32) {
        const int s = gr.s0 + j;
        const double bb = row_total(part, 0, s, G.nsys, gridDim.x);
        const double rz = row_total(part, 1, s, G.nsys, gridDim.x);
        const double rr = row_total(part, 2, s, G.nsys, gridDim.x);
        if (lane != 0) continue;
        const double bn = sqrt(bb);
        const double rel = bn > 0.0 ? sqrt(rr) / bn : 0.0;
        const bool finite = isfinite(bn) && isfinite(rz) && isfinite(rr);
        int act = bn > 0.0 && finite;
        if (act && precheck && rel <= tol) act = 0;
        sc.bn[s] = bn;
        sc.rz[s] = rz;
        sc.rr[s] = rr;
        sc.alpha[s] = 0.0;
        sc.beta[s] = 0.0;
        sc.act[s] = act;
        sc.iters[s] = 0;
        sc.relres[s] = rel;
        sc.status[s] = finite ? LPM_STATUS_OK : LPM_STATUS_BREAKDOWN;
        if (!act) atomicAdd(sc.nconv, 1u);
    }
    if (threadIdx.x == 0) cnt[gr.gid] = 0u;
}

// ----------------------------------------------------------------------------------------------------- update
template <typename T, bool PREC, bool PAIRED>
__global__ void __launch_bounds__(VB) k_fcg_update(VecGeom G, int it, int check, int maxit, double tol,
                                                   const uint8_t* __restrict__ mask, const T* __restrict__ Ms,
                                                   T* __restrict__ r, const T* __restrict__ Ap, FcgScalars sc,
                                                   double* part, unsigned* cnt)
{
    __shared__ double sh[GRP * 2 * 8];
    __shared__ bool last;
    const Group gr = group_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    double vals[GRP][2];
    T m9[9];
    bool any = false;
    for (int j = 0; j < gr.nsg; ++j) any |= sc.act[gr.s0 + j] != 0;
    if (PREC && any && i < N) {
#pragma unroll
        for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)gr.set * 9 + e) * N + i];
    }
#pragma unroll
    for (int j = 0; j < GRP; ++j) {
        vals[j][0] = vals[j][1] = 0.0;
        if (j >= gr.nsg || i >= N) continue;
        const int s = gr.s0 + j;
        if (!sc.act[s]) continue;
        const int64_t o = ((int64_t)s * N + i) * 3;
        const T al = (T)sc.alpha[s];
        const uint8_t* m = mask ? mask + ((int64_t)(s % G.nmask) * N + i) * 3 : nullptr;
        T rv[3], zv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T ap = (m && !m[a]) ? T(0) : Ap[vix<PAIRED>(G, s, i, a)];
            rv[a] = r[o + a] - al * ap;
            r[o + a] = rv[a];
        }
        precond<T, PREC>(m9, m, rv, zv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            vals[j][0] += (double)rv[a] * (double)zv[a];
            vals[j][1] += (double)rv[a] * (double)rv[a];
        }
    }
    if (!group_reduce<2>(vals, gr.nsg, gr.s0, G.nsys, part, cnt, gr.gid, sh, &last)) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cur = (it - 1) & 1, nxt = it & 1;
    for (int j = w; j < gr.nsg; j += VB / 32) {
        const int s = gr.s0 + j;
        const double rzn = row_total(part, 0, s, G.nsys, gridDim.x);
        const double rrn = row_total(part, 1, s, G.nsys, gridDim.x);
        if (lane != 0 || !sc.act[s]) continue;
        const double rzc = sc.rz[cur * G.nsys + s];
        sc.rz[nxt * G.nsys + s] = rzn;
        sc.rr[s] = rrn;
        sc.beta[s] = rzc != 0.0 ? rzn / rzc : 0.0;
        const double rel = sqrt(rrn) / sc.bn[s];
        if (!isfinite(rrn) || !isfinite(rzn)) {
            sc.act[s] = 0;
            sc.iters[s] = it;
            sc.relres[s] = rel;
            sc.status[s] = LPM_STATUS_BREAKDOWN;
            atomicAdd(sc.nconv, 1u);
            continue;
        }
        if (it % check == 0 || it == maxit) {
            sc.relres[s] = rel;
            if (rel <= tol || it == maxit) {
                sc.act[s] = 0;
                sc.iters[s] = it;
                if (rel > tol) sc.status[s] = LPM_STATUS_NOT_CONVERGED;
                atomicAdd(sc.nconv, 1u);
            }
        }
    }
    if (threadIdx.x == 0) cnt[gr.gid] = 0u;
}

// --------------------------------------------------------------------------------------------------- p-update
template <typename T, bool PREC, bool PAIRED>
__global__ void __launch_bounds__(VB) k_fcg_pupdate(VecGeom G, const uint8_t* __restrict__ mask,
                                                    const T* __restrict__ Ms, T* __restrict__ x,
                                                    const T* __restrict__ r, T* __restrict__ p, FcgScalars sc)
{
    const Group gr = group_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    T m9[9];
    bool loaded = false;
#pragma unroll
    for (int j = 0; j < GRP; ++j) {
        if (j >= gr.nsg) break;
        const int s = gr.s0 + j;
        const double alpha = sc.alpha[s];
        const int act = sc.act[s];
        if (alpha == 0.0 && !act) continue;
        const int64_t o = ((int64_t)s * N + i) * 3;
        T pv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) pv[a] = p[vix<PAIRED>(G, s, i, a)];
        if (alpha != 0.0) {
            const T al = (T)alpha;
#pragma unroll
            for (int a = 0; a < 3; ++a) x[o + a] += al * pv[a];
        }
        if (!act) continue;
        if (PREC && !loaded) {
#pragma unroll
            for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)gr.set * 9 + e) * N + i];
            loaded = true;
        }
        T rv[3], zv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) rv[a] = r[o + a];
        precond<T, PREC>(m9, mask ? mask + ((int64_t)(s % G.nmask) * N + i) * 3 : nullptr, rv, zv);
        const T be = (T)sc.beta[s];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[vix<PAIRED>(G, s, i, a)] = zv[a] + be * pv[a];
    }
}

inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

struct Carve {
    char* base;
    size_t off;
    template <typename X>
    X* take(size_t n)
    {
        X* q = base ? reinterpret_cast<X*>(base + off) : nullptr;
        off = align_up(off + n * sizeof(X));
        return q;
    }
};

template <typename T>
struct FWork {
    T *r, *p, *Ap, *Ms;
    FcgScalars sc;
    double *vpart, *mpart;
    unsigned *vcnt, *mcnt;
    int* err;
};

// FP32 boxes run the pair-packed operator (p and Ap in the pair layout); FP64 the TMA operator.
template <typename T>
bool use_pairs(const Lattice& L)
{
    return sizeof(T) == 4 && pair_supported(L.nx);
}

template <typename T>
void carve(Carve& c, const Lattice& L, int nsys, int rps, bool precond, FWork<T>& w)
{
    const int nset = (nsys + rps - 1) / rps;
    const int npp = (rps + 1) / 2;
    const bool paired = use_pairs<T>(L);
    const size_t nv = (size_t)nsys * L.N * 3;
    const size_t nvp = paired ? (size_t)nset * npp * L.N * 6 : nv;
    const int nb = (int)((L.N + VB - 1) / VB);
    const int dots = paired ? pair_dot_blocks_max(L.nx, L.ny, L.nz)
                            : tma_dot_blocks_max(L.nx, L.ny, L.nz, (int)sizeof(T));
    w.r = c.take<T>(nv);
    w.p = c.take<T>(nvp);
    w.Ap = c.take<T>(nvp);
    w.Ms = precond ? c.take<T>((size_t)nset * 9 * L.N) : nullptr;
    w.sc.nsys = nsys;
    w.sc.bn = c.take<double>(nsys);
    w.sc.rz = c.take<double>(2 * (size_t)nsys);
    w.sc.rr = c.take<double>(nsys);
    w.sc.pAp = c.take<double>(nsys);
    w.sc.alpha = c.take<double>(nsys);
    w.sc.beta = c.take<double>(nsys);
    w.sc.act = c.take<int>(nsys);
    w.sc.nconv = c.take<unsigned>(1);
    w.vpart = c.take<double>((size_t)3 * nsys * nb);
    w.vcnt = c.take<unsigned>((size_t)nset * ((rps + GRP - 1) / GRP) + 1);
    w.mpart = c.take<double>((size_t)nsys * dots);
    w.mcnt = c.take<unsigned>(nsys);
    w.err = c.take<int>(1);
}

// One operator launch: out = K u, with the alpha-step epilogue when epi.
template <typename T>
struct Operator {
    bool paired;
    TmaArgs<T> ta;
    PairArgs pa;
    cudaError_t run(const T* u, T* out, bool epi, int it, cudaStream_t st)
    {
        if constexpr (sizeof(T) == 4) {
            if (paired) {
                PairArgs a = pa;
                a.u = u;
                a.out = out;
                a.it = it;
                if (!epi) {
                    a.act = nullptr;
                    a.part = nullptr;
                    a.has_sc = 0;
                }
                return launch_sc_pair(a, epi, st);
            }
        }
        TmaArgs<T> a = ta;
        a.u = u;
        a.out = out;
        a.it = it;
        if (!epi) {
            a.mask = nullptr;
            a.act = nullptr;
            a.part = nullptr;
            a.has_sc = 0;
        }
        return launch_sc_tma<T>(a, epi, st);
    }
};

template <typename T, bool PREC, bool PAIRED>
void launch_vec_init(dim3 vg, cudaStream_t st, const VecGeom& G, const T* b, const T* Ax, const uint8_t* mask,
                     FWork<T>& w, double tol, int precheck)
{
    k_fcg_init<T, PREC, PAIRED><<<vg, VB, 0, st>>>(G, b, Ax, mask, w.Ms, w.r, w.p, w.sc, w.vpart, w.vcnt, tol,
                                                    precheck);
}

template <typename T, bool PREC, bool PAIRED>
void launch_vec_iter(dim3 vg, cudaStream_t st, const VecGeom& G, int it, const lpm_cg_opts& o, const uint8_t* mask,
                     T* x, FWork<T>& w)
{
    k_fcg_update<T, PREC, PAIRED><<<vg, VB, 0, st>>>(G, it, o.check, o.maxit, o.tol, mask, w.Ms, w.r, w.Ap, w.sc,
                                                      w.vpart, w.vcnt);
    k_fcg_pupdate<T, PREC, PAIRED><<<vg, VB, 0, st>>>(G, mask, w.Ms, x, w.r, w.p, w.sc);
}

}  // namespace

size_t cg_fused_workspace_bytes(const Lattice& L, int nsys, int rhs_per_set, int elem_bytes, int precond)
{
    Carve c{nullptr, 0};
    if (elem_bytes == 4) {
        FWork<float> w;
        carve<float>(c, L, nsys, rhs_per_set, precond != 0, w);
    } else {
        FWork<double> w;
        carve<double>(c, L, nsys, rhs_per_set, precond != 0, w);
    }
    return c.off + 256;
}

template <typename T>
int cg_solve_fused(const Lattice& L, const T* Kn, const T* Tv, const Batch& bt, const T* Minv, const uint8_t* mask,
                   const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws, size_t ws_bytes, int* iters,
                   double* relres, int* status, cudaStream_t st)
{
    if (o.maxit < 0 || o.check < 1 || o.poll < 1 || bt.nsys < 1) return LPM_ERR_ARG;
    const bool precond = Minv != nullptr;
    char* base = static_cast<char*>(ws);
    const size_t shift = (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    Carve c{base + shift, 0};
    FWork<T> w;
    carve<T>(c, L, bt.nsys, bt.rhs_per_set, precond, w);
    if (c.off + shift > ws_bytes) return LPM_ERR_WORKSPACE;
    w.sc.iters = iters;
    w.sc.relres = relres;
    w.sc.status = status;
    const int64_t N = L.N;
    const int nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    const int vgrp = (bt.rhs_per_set + GRP - 1) / GRP;
    const int npp = (bt.rhs_per_set + 1) / 2;
    const bool paired = use_pairs<T>(L);
    const VecGeom G{N, bt.nsys, bt.rhs_per_set, bt.nmask, vgrp, npp};
    const int nb = (int)((N + VB - 1) / VB);
    cudaError_t e = cudaMemsetAsync(w.vcnt, 0, sizeof(unsigned) * (nset * vgrp + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mcnt, 0, sizeof(unsigned) * bt.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.sc.nconv, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.err, 0, sizeof(int), st);
    if (e == cudaSuccess && paired)  // dummy lanes of the pair layout stay zero
        e = cudaMemsetAsync(w.p, 0, sizeof(T) * (size_t)nset * npp * N * 6, st);
    if (e != cudaSuccess) return (int)e;
    if (precond) k_repack_M<T><<<dim3(nb, nset), VB, 0, st>>>(Minv, w.Ms, N);

    Operator<T> op{};
    op.paired = paired;
    if (paired) {
        PairArgs& a = op.pa;
        a.nx = L.nx;
        a.ny = L.ny;
        a.nz = L.nz;
        a.N = N;
        a.nsys = bt.nsys;
        a.rhs_per_set = bt.rhs_per_set;
        a.npp = npp;
        a.npair = nset * npp;
        a.zchunk = pair_zchunk(L.nx, L.ny, L.nz, a.npair);
        a.Kn = reinterpret_cast<const float*>(Kn);
        a.Tv = reinterpret_cast<const float*>(Tv);
        a.act = w.sc.act;
        a.part = w.mpart;
        a.cnt = w.mcnt;
        a.scv = w.sc;
        a.has_sc = 1;
        a.err = w.err;
    } else {
        TmaArgs<T>& a = op.ta;
        a.nx = L.nx;
        a.ny = L.ny;
        a.nz = L.nz;
        a.N = N;
        a.nsys = bt.nsys;
        a.rhs_per_set = bt.rhs_per_set;
        a.nmask = bt.nmask;
        tma_configure(a);
        a.Kn = Kn;
        a.Tv = Tv;
        a.mask = mask;
        a.act = w.sc.act;
        a.part = w.mpart;
        a.cnt = w.mcnt;
        a.scv = w.sc;
        a.has_sc = 1;
        a.err = w.err;
    }
    if (!x_is_zero) {
        const T* xin = x;
        if (paired) {
            if constexpr (sizeof(T) == 4) {
                if ((e = pair_pack(x, w.p, N, bt.nsys, bt.rhs_per_set, st)) != cudaSuccess) return (int)e;
                xin = w.p;
            }
        }
        if ((e = op.run(xin, w.Ap, false, 0, st)) != cudaSuccess) return (int)e;
    }
    const dim3 vg(nb, nset * vgrp);
    const T* Ax = x_is_zero ? nullptr : w.Ap;
    if (precond)
        paired ? launch_vec_init<T, true, true>(vg, st, G, b, Ax, mask, w, o.tol, o.precheck)
               : launch_vec_init<T, true, false>(vg, st, G, b, Ax, mask, w, o.tol, o.precheck);
    else
        paired ? launch_vec_init<T, false, true>(vg, st, G, b, Ax, mask, w, o.tol, o.precheck)
               : launch_vec_init<T, false, false>(vg, st, G, b, Ax, mask, w, o.tol, o.precheck);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    unsigned nconv = 0;
    e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;

    KmvTimer timer(o.prof, st);
    int rc = LPM_OK;
    for (int it = 1; it <= o.maxit && nconv < (unsigned)bt.nsys; ++it) {
        timer.begin(nconv == 0);
        e = op.run(w.p, w.Ap, true, it, st);
        timer.end();
        if (e != cudaSuccess) return (int)e;
        if (precond)
            paired ? launch_vec_iter<T, true, true>(vg, st, G, it, o, mask, x, w)
                   : launch_vec_iter<T, true, false>(vg, st, G, it, o, mask, x, w);
        else
            paired ? launch_vec_iter<T, false, true>(vg, st, G, it, o, mask, x, w)
                   : launch_vec_iter<T, false, false>(vg, st, G, it, o, mask, x, w);
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        if (it % o.poll == 0 || it == o.maxit) {
            e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return (int)e;
            timer.collect();
        }
    }
    timer.collect();
    int err = 0;
    e = cudaMemcpyAsync(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    if (err) rc = LPM_ERR_TIMEOUT;
    return rc;
}

template int cg_solve_fused<float>(const Lattice&, const float*, const float*, const Batch&, const float*,
                                   const uint8_t*, const float*, float*, int, const lpm_cg_opts&, void*, size_t, int*,
                                   double*, int*, cudaStream_t);
template int cg_solve_fused<double>(const Lattice&, const double*, const double*, const Batch&, const double*,
                                    const uint8_t*, const double*, double*, int, const lpm_cg_opts&, void*, size_t,
                                    int*, double*, int*, cudaStream_t);

}  // namespace lpm
