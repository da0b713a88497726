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
#include <cstring>
#include <map>
#include <mutex>

#include "lpm_graph.h"
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
    int npp;   // pairs per set (pair layout)
};

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
template <int NV, int GS = GRP, typename A = double>
__device__ __forceinline__ bool group_reduce(A (*vals)[NV], int nsg, int s0, int nsys, double* part, unsigned* cnt,
                                             int gid, double* sh, bool* last)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < GS; ++j) {
        if (j >= nsg) break;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double t = warp_sum((double)vals[j][v]);
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
template <typename T, bool PREC>
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
            T w = Ax ? bv - Ax[o + a] : bv;
            if (m && !m[a]) w = T(0);
            rv[a] = w;
            vals[j][0] += (double)bv * (double)bv;
        }
        precond<T, PREC>(m9, m, rv, zv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            r[o + a] = rv[a];
            p[o + a] = zv[a];
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
        if (act && precheck && rel <= (sc.tols ? sc.tols[s] : tol)) act = 0;
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

// Last block of a system group after the r.z / r.r reduction: beta, convergence test every `check` iterations,
// freezing of converged or broken-down systems.
__device__ __forceinline__ void update_tail(const VecGeom& G, const Group& gr, int it, int check, int maxit,
                                            double tol, FcgScalars& sc, const double* part, unsigned* cnt)
{
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
        const double tl = sc.tols ? sc.tols[s] : tol;
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
            if (rel <= tl || it == maxit) {
                sc.act[s] = 0;
                sc.iters[s] = it;
                if (rel > tl) sc.status[s] = LPM_STATUS_NOT_CONVERGED;
                atomicAdd(sc.nconv, 1u);
            }
        }
    }
    if (threadIdx.x == 0) cnt[gr.gid] = 0u;
}

// ----------------------------------------------------------------------------------------------------- update
template <typename T, bool PREC>
__global__ void __launch_bounds__(VB) k_fcg_update(VecGeom G, int it_host, int check, int maxit, double tol,
                                                   const uint8_t* __restrict__ mask, const T* __restrict__ Ms,
                                                   T* __restrict__ r, const T* __restrict__ Ap, FcgScalars sc,
                                                   double* part, unsigned* cnt)
{
    const int it = sc.itp ? *sc.itp : it_host;
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
    // one system: r -= alpha mask(Ap); z = mask(M r); accumulate r.z, r.r
    auto one = [&](int s, const T* ap, int stride, double* v) {
        const int64_t o = ((int64_t)s * N + i) * 3;
        const T al = (T)sc.alpha[s];
        const uint8_t* m = mask ? mask + ((int64_t)(s % G.nmask) * N + i) * 3 : nullptr;
        T rv[3], zv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T apv = (m && !m[a]) ? T(0) : ap[a * stride];
            rv[a] = r[o + a] - al * apv;
            r[o + a] = rv[a];
        }
        precond<T, PREC>(m9, m, rv, zv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            v[0] += (double)rv[a] * (double)zv[a];
            v[1] += (double)rv[a] * (double)rv[a];
        }
    };
#pragma unroll
    for (int j = 0; j < GRP; ++j) vals[j][0] = vals[j][1] = 0.0;
    if (i < N) {
#pragma unroll
        for (int j = 0; j < GRP; ++j) {
            if (j >= gr.nsg) break;
            const int s = gr.s0 + j;
            if (!sc.act[s]) continue;
            one(s, Ap + ((int64_t)s * N + i) * 3, 1, vals[j]);
        }
    }
    if (!group_reduce<2>(vals, gr.nsg, gr.s0, G.nsys, part, cnt, gr.gid, sh, &last)) return;
    update_tail(G, gr, it, check, maxit, tol, sc, part, cnt);
}

// --------------------------------------------------------------------------------------------------- p-update
template <typename T, bool PREC>
__global__ void __launch_bounds__(VB) k_fcg_pupdate(VecGeom G, const uint8_t* __restrict__ mask,
                                                    const T* __restrict__ Ms, T* __restrict__ x,
                                                    const T* __restrict__ r, T* __restrict__ p, FcgScalars sc)
{
    if (sc.itp && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(sc.itp, 1);
    const Group gr = group_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    T m9[9];
    bool loaded = false;
    // one system: x += alpha p; p = mask(M r) + beta p (active systems); p values at pv[a * stride]
    auto one = [&](int s, T* pv, int stride) -> bool {
        const double alpha = sc.alpha[s];
        const int act = sc.act[s];
        if (alpha == 0.0 && !act) return false;
        const int64_t o = ((int64_t)s * N + i) * 3;
        if (alpha != 0.0) {
            const T al = (T)alpha;
#pragma unroll
            for (int a = 0; a < 3; ++a) x[o + a] += al * pv[a * stride];
        }
        if (!act) return false;
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
        for (int a = 0; a < 3; ++a) pv[a * stride] = zv[a] + be * pv[a * stride];
        return true;
    };
#pragma unroll
    for (int j = 0; j < GRP; ++j) {
        if (j >= gr.nsg) break;
        const int s = gr.s0 + j;
        if (sc.alpha[s] == 0.0 && !sc.act[s]) continue;
        T* pp = p + ((int64_t)s * N + i) * 3;
        T pv[3] = {pp[0], pp[1], pp[2]};
        if (one(s, pv, 1)) {
            pp[0] = pv[0];
            pp[1] = pv[1];
            pp[2] = pv[2];
        }
    }
}

// ------------------------------------------------------------------------------- FP32 pair-layout kernels
// In FP32 every vector of the engine (r, x, p, Ap) lives in the pair layout; a thread handles one particle of one
// pair (both systems: 24 contiguous bytes per vector), a block row one pair.  The 3x3 preconditioner blocks of a set
// are read by the blocks of its pairs at about the same time (adjacent grid rows), so they come from L2 after the
// first.  b and x cross the solve boundary in the (nsys, N, 3) layout.
struct PairSys {
    int pr, set, s0, nl;  // pair, set, first system, real lanes (1 or 2)
};

__device__ __forceinline__ PairSys pair_of(const VecGeom& G)
{
    PairSys q;
    q.pr = blockIdx.y;
    q.set = q.pr / G.npp;
    const int jp = q.pr - q.set * G.npp;
    q.s0 = q.set * G.rps + 2 * jp;
    q.nl = min(2, min(G.rps - 2 * jp, G.nsys - q.s0));
    return q;
}

__device__ __forceinline__ unsigned mask_bits(const uint8_t* mask, const VecGeom& G, int s, int64_t i)
{
    if (!mask) return 7u;
    const uint8_t* m = mask + ((int64_t)(s % G.nmask) * G.N + i) * 3;
    return (m[0] ? 1u : 0u) | (m[1] ? 2u : 0u) | (m[2] ? 4u : 0u);
}

template <bool PREC>
__device__ __forceinline__ void precond_bits(const float* m9, unsigned mb, const float* rv, float* zv)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float z = PREC ? m9[3 * a] * rv[0] + m9[3 * a + 1] * rv[1] + m9[3 * a + 2] * rv[2] : rv[a];
        zv[a] = ((mb >> a) & 1u) ? z : 0.f;
    }
}

// v[l][a] <-> 6 contiguous floats (a, lane)
__device__ __forceinline__ void ld_pair(const float* src, float (*v)[3])
{
    const float2* q = reinterpret_cast<const float2*>(src);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float2 t = q[a];
        v[0][a] = t.x;
        v[1][a] = t.y;
    }
}
__device__ __forceinline__ void st_pair(float* dst, const float (*v)[3])
{
    float2* q = reinterpret_cast<float2*>(dst);
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = make_float2(v[0][a], v[1][a]);
}

// r = mask(b - Ax), p = z = mask(M r); b.b, r.z, r.r per system; dummy lanes written as zero.
template <bool PREC>
__global__ void __launch_bounds__(VB) k_pair_init(VecGeom G, const float* __restrict__ b, const float* __restrict__ Ax,
                                                  const uint8_t* __restrict__ mask, const float* __restrict__ Ms,
                                                  float* __restrict__ r, float* __restrict__ p, FcgScalars sc,
                                                  double* part, unsigned* cnt, double tol, int precheck)
{
    __shared__ double sh[2 * 3 * 8];
    __shared__ bool last;
    const PairSys q = pair_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    float vals[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    if (i < N) {
        const int64_t po = ((int64_t)q.pr * N + i) * 6;
        float ax[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, rv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}},
              zv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, m9[9];
        if (Ax) ld_pair(Ax + po, ax);
        if (PREC) {
#pragma unroll
            for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)q.set * 9 + e) * N + i];
        }
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            if (l >= q.nl) break;
            const int s = q.s0 + l;
            const unsigned mb = mask_bits(mask, G, s, i);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float bv = b[((int64_t)s * N + i) * 3 + a];
                rv[l][a] = ((mb >> a) & 1u) ? bv - ax[l][a] : 0.f;
                vals[l][0] += bv * bv;
            }
            precond_bits<PREC>(m9, mb, rv[l], zv[l]);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                vals[l][1] += rv[l][a] * zv[l][a];
                vals[l][2] += rv[l][a] * rv[l][a];
            }
        }
        st_pair(r + po, rv);
        st_pair(p + po, zv);
    }
    if (!group_reduce<3, 2, float>(vals, q.nl, q.s0, G.nsys, part, cnt, q.pr, sh, &last)) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = w; j < q.nl; j += VB / 32) {
        const int s = q.s0 + j;
        const double bb = row_total(part, 0, s, G.nsys, gridDim.x);
        const double rz = row_total(part, 1, s, G.nsys, gridDim.x);
        const double rr = row_total(part, 2, s, G.nsys, gridDim.x);
        if (lane != 0) continue;
        const double bn = sqrt(bb);
        const double rel = bn > 0.0 ? sqrt(rr) / bn : 0.0;
        const bool finite = isfinite(bn) && isfinite(rz) && isfinite(rr);
        int act = bn > 0.0 && finite;
        if (act && precheck && rel <= (sc.tols ? sc.tols[s] : tol)) act = 0;
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
    if (threadIdx.x == 0) cnt[q.pr] = 0u;
}

// r -= alpha mask(Ap); z = mask(M r); r.z, r.r; the last block of the pair forms beta and tests convergence.
template <bool PREC>
__global__ void __launch_bounds__(VB) k_pair_update(VecGeom G, int it_host, int check, int maxit, double tol,
                                                    const uint8_t* __restrict__ mask, const float* __restrict__ Ms,
                                                    float* __restrict__ r, const float* __restrict__ Ap,
                                                    FcgScalars sc, double* part, unsigned* cnt)
{
    const int it = sc.itp ? *sc.itp : it_host;
    __shared__ double sh[2 * 2 * 8];
    __shared__ bool last;
    const PairSys q = pair_of(G);
    const int64_t N = G.N;
    // q.nl < 1: a pair of a trailing partial set with no system behind it
    const bool act0 = q.nl > 0 && sc.act[q.s0] != 0, act1 = q.nl > 1 && sc.act[q.s0 + 1] != 0;
    float vals[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
    // grid-stride over particles: few blocks per pair, so the reduction epilogue (fence, counter) is amortised
    for (int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x; i < N && (act0 || act1); i += (int64_t)gridDim.x * VB) {
        const int64_t po = ((int64_t)q.pr * N + i) * 6;
        float ap[2][3], rv[2][3], m9[9];
        ld_pair(Ap + po, ap);
        ld_pair(r + po, rv);
        if (PREC) {
#pragma unroll
            for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)q.set * 9 + e) * N + i];
        }
        const unsigned mb0 = act0 ? mask_bits(mask, G, q.s0, i) : 0u;
        const unsigned mb1 = act1 ? mask_bits(mask, G, q.s0 + 1, i) : 0u;
        const float al0 = (float)sc.alpha[q.s0], al1 = act1 ? (float)sc.alpha[q.s0 + 1] : 0.f;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const bool on = l ? act1 : act0;
            if (!on) continue;
            const unsigned mb = l ? mb1 : mb0;
            const float al = l ? al1 : al0;
            float zv[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) rv[l][a] -= ((mb >> a) & 1u) ? al * ap[l][a] : 0.f;
            precond_bits<PREC>(m9, mb, rv[l], zv);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                vals[l][0] += rv[l][a] * zv[a];
                vals[l][1] += rv[l][a] * rv[l][a];
            }
        }
        st_pair(r + po, rv);
    }
    Group gr;
    gr.gid = q.pr;
    gr.set = q.set;
    gr.s0 = q.s0;
    gr.nsg = q.nl;
    if (!group_reduce<2, 2, float>(vals, q.nl, q.s0, G.nsys, part, cnt, q.pr, sh, &last)) return;
    update_tail(G, gr, it, check, maxit, tol, sc, part, cnt);
}

// x += alpha p; p = mask(M r) + beta p (active systems).
template <bool PREC>
__global__ void __launch_bounds__(VB) k_pair_pupdate(VecGeom G, const uint8_t* __restrict__ mask,
                                                     const float* __restrict__ Ms, float* __restrict__ x,
                                                     const float* __restrict__ r, float* __restrict__ p,
                                                     FcgScalars sc)
{
    if (sc.itp && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(sc.itp, 1);
    const PairSys q = pair_of(G);
    const int64_t N = G.N;
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    const bool two = q.nl > 1;
    const bool one = q.nl > 0;  // false for a pair of a trailing partial set with no system behind it
    const double a0d = one ? sc.alpha[q.s0] : 0.0, a1d = two ? sc.alpha[q.s0 + 1] : 0.0;
    const bool act0 = one && sc.act[q.s0] != 0, act1 = two && sc.act[q.s0 + 1] != 0;
    const bool mov = a0d != 0.0 || a1d != 0.0;
    if (!mov && !act0 && !act1) return;
    const int64_t po = ((int64_t)q.pr * N + i) * 6;
    float pv[2][3], xv[2][3], rv[2][3], m9[9];
    ld_pair(p + po, pv);
    if (mov) ld_pair(x + po, xv);
    if (act0 || act1) {
        ld_pair(r + po, rv);
        if (PREC) {
#pragma unroll
            for (int e = 0; e < 9; ++e) m9[e] = Ms[((int64_t)q.set * 9 + e) * N + i];
        }
    }
    if (mov) {
        const float al[2] = {(float)a0d, (float)a1d};
#pragma unroll
        for (int l = 0; l < 2; ++l)
#pragma unroll
            for (int a = 0; a < 3; ++a) xv[l][a] += al[l] * pv[l][a];
        st_pair(x + po, xv);
    }
    if (act0 || act1) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const bool on = l ? act1 : act0;
            if (!on) continue;
            const int s = q.s0 + l;
            float zv[3];
            precond_bits<PREC>(m9, mask_bits(mask, G, s, i), rv[l], zv);
            const float be = (float)sc.beta[s];
#pragma unroll
            for (int a = 0; a < 3; ++a) pv[l][a] = zv[a] + be * pv[l][a];
        }
        st_pair(p + po, pv);
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
    T *r, *p, *Ap, *Ms, *xp;  // xp: pair-layout x (FP32 path)
    FcgScalars sc;
    double *vpart, *mpart;
    unsigned *vcnt, *mcnt;
    int* err;
};

// FP32 boxes run the pair-packed operator with every engine vector in the pair layout; FP64 the TMA operator.
template <typename T>
bool use_pairs(const Lattice& L)
{
    return sizeof(T) == 4 && pair_supported(L.nx);
}

// FP64 systems on the FP64 instantiation of the pair operator (natural layout; p stays zero on fixed DOFs, so its
// unmasked p.Ap is the masked one).
template <typename T>
bool use_pair64(const Lattice& L)
{
    return sizeof(T) == 8 && pair64_supported(L.nx);
}

template <typename T>
void carve(Carve& c, const Lattice& L, int nsys, int rps, bool precond, FWork<T>& w)
{
    const int nset = (nsys + rps - 1) / rps;
    const int npp = (rps + 1) / 2;
    const bool paired = use_pairs<T>(L);
    const size_t nv = paired ? (size_t)nset * npp * L.N * 6 : (size_t)nsys * L.N * 3;
    const int nb = (int)((L.N + VB - 1) / VB);
    const int dots = (paired || use_pair64<T>(L)) ? pair_dot_blocks_max(L.nx, L.ny, L.nz)
                                                  : tma_dot_blocks_max(L.nx, L.ny, L.nz, (int)sizeof(T));
    w.r = c.take<T>(nv);
    w.p = c.take<T>(nv);
    w.Ap = c.take<T>(nv);
    w.xp = paired ? c.take<T>(nv) : nullptr;
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
    w.vcnt = c.take<unsigned>((size_t)nset * rps + 1);  // one per group or pair
    w.mpart = c.take<double>((size_t)nsys * dots);
    w.mcnt = c.take<unsigned>(nsys);
    w.err = c.take<int>(1);
    w.sc.itp = c.take<int>(1);
}

// One operator launch: out = K u, with the alpha-step epilogue when epi.
template <typename T>
struct Operator {
    bool paired;  // FP32 pair layout
    bool p64;     // FP64 pair operator on natural-layout vectors
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
        } else {
            if (p64) {
                PairArgs a = pa;
                a.u = reinterpret_cast<const float*>(u);
                a.out = reinterpret_cast<float*>(out);
                a.it = it;
                if (!epi) {
                    a.act = nullptr;
                    a.part = nullptr;
                    a.has_sc = 0;
                }
                return launch_sc_pair64(a, epi, st);
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

// Vector kernels of one engine step (init, or update + p-update) in the layout of the path.
template <typename T, bool PREC>
void launch_init(bool paired, dim3 vg, dim3 pg, cudaStream_t st, const VecGeom& G, const T* b, const T* Ax,
                 const uint8_t* mask, FWork<T>& w, double tol, int precheck)
{
    if constexpr (sizeof(T) == 4) {
        if (paired) {
            k_pair_init<PREC><<<pg, VB, 0, st>>>(G, b, Ax, mask, w.Ms, w.r, w.p, w.sc, w.vpart, w.vcnt, tol, precheck);
            return;
        }
    }
    k_fcg_init<T, PREC><<<vg, VB, 0, st>>>(G, b, Ax, mask, w.Ms, w.r, w.p, w.sc, w.vpart, w.vcnt, tol, precheck);
}

template <typename T, bool PREC>
void launch_iter(bool paired, dim3 vg, dim3 pg, cudaStream_t st, const VecGeom& G, int it, const lpm_cg_opts& o,
                 const uint8_t* mask, T* x, FWork<T>& w)
{
    if constexpr (sizeof(T) == 4) {
        if (paired) {
            // about two waves of blocks (4 resident per SM) for the reducing kernel
            const unsigned gx = std::max(1u, std::min(pg.x, (unsigned)((2 * 4 * 148 + pg.y - 1) / pg.y)));
            k_pair_update<PREC><<<dim3(gx, pg.y), VB, 0, st>>>(G, it, o.check, o.maxit, o.tol, mask, w.Ms, w.r, w.Ap,
                                                               w.sc, w.vpart, w.vcnt);
            k_pair_pupdate<PREC><<<pg, VB, 0, st>>>(G, mask, w.Ms, w.xp, w.r, w.p, w.sc);
            return;
        }
    }
    k_fcg_update<T, PREC><<<vg, VB, 0, st>>>(G, it, o.check, o.maxit, o.tol, mask, w.Ms, w.r, w.Ap, w.sc, w.vpart,
                                             w.vcnt);
    k_fcg_pupdate<T, PREC><<<vg, VB, 0, st>>>(G, mask, w.Ms, x, w.r, w.p, w.sc);
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
    w.sc.tols = o.tol_sys;
    const int64_t N = L.N;
    const int nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    const int vgrp = (bt.rhs_per_set + GRP - 1) / GRP;
    const int npp = (bt.rhs_per_set + 1) / 2;
    const bool paired = use_pairs<T>(L);
    if (paired && nset * npp > 65535) return LPM_ERR_UNSUPPORTED;
    const VecGeom G{N, bt.nsys, bt.rhs_per_set, bt.nmask, vgrp, npp};
    const int nb = (int)((N + VB - 1) / VB);
    const size_t nvp = (size_t)nset * npp * N * 6;
    cudaError_t e = cudaMemsetAsync(w.vcnt, 0, sizeof(unsigned) * ((size_t)nset * bt.rhs_per_set + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mcnt, 0, sizeof(unsigned) * bt.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.sc.nconv, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.err, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (precond) k_repack_M<T><<<dim3(nb, nset), VB, 0, st>>>(Minv, w.Ms, N);

    Operator<T> op{};
    op.paired = paired;
    op.p64 = use_pair64<T>(L);
    if (op.p64) {
        PairArgs& a = op.pa;
        a = pair64_args(L.nx, L.ny, L.nz, N, bt.nsys, bt.rhs_per_set, reinterpret_cast<const double*>(x),
                        reinterpret_cast<const double*>(Kn), reinterpret_cast<const double*>(Tv),
                        reinterpret_cast<double*>(w.Ap));
        a.act = w.sc.act;
        a.part = w.mpart;
        a.cnt = w.mcnt;
        a.scv = w.sc;
        a.has_sc = 1;
        a.err = w.err;
    } else if (paired) {
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
        a.variant = pair_variant(L.nx, L.ny, L.nz, a.npair);
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
    // start vector: x (natural layout), or its pair-layout copy xp that the FP32 engine updates
    if constexpr (sizeof(T) == 4) {
        if (paired) {
            e = x_is_zero ? cudaMemsetAsync(w.xp, 0, sizeof(T) * nvp, st)
                          : pair_pack(x, w.xp, N, bt.nsys, bt.rhs_per_set, st);
            if (e != cudaSuccess) return (int)e;
        }
    }
    if (!x_is_zero)
        if ((e = op.run(paired ? w.xp : x, w.Ap, false, 0, st)) != cudaSuccess) return (int)e;
    const dim3 vg(nb, nset * vgrp), pg(nb, nset * npp);
    const T* Ax = x_is_zero ? nullptr : w.Ap;
    if (precond)
        launch_init<T, true>(paired, vg, pg, st, G, b, Ax, mask, w, o.tol, o.precheck);
    else
        launch_init<T, false>(paired, vg, pg, st, G, b, Ax, mask, w, o.tol, o.precheck);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    unsigned nconv = 0;
    e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;

    KmvTimer timer(o.prof, st);
    int rc = LPM_OK;
    static const int kOne = 1;
    if ((e = cudaMemcpyAsync(w.sc.itp, &kOne, sizeof(int), cudaMemcpyHostToDevice, st)) != cudaSuccess) return (int)e;
    auto one_iter = [&](int it, cudaStream_t s) -> cudaError_t {
        timer.begin(nconv == 0);
        cudaError_t ee = op.run(w.p, w.Ap, true, it, s);
        timer.end();
        if (ee != cudaSuccess) return ee;
        if (precond)
            launch_iter<T, true>(paired, vg, pg, s, G, it, o, mask, x, w);
        else
            launch_iter<T, false>(paired, vg, pg, s, G, it, o, mask, x, w);
        return cudaGetLastError();
    };
    GraphKey key;
    key.ptr = {ws, Kn, Tv, mask, x, o.tol_sys, nullptr, nullptr, nullptr, nullptr};
    key.val = {1, bt.nsys, bt.rhs_per_set, bt.nmask, L.nx, L.ny, L.nz, o.poll, o.check, o.maxit, precond ? 1 : 0,
               (long long)sizeof(T), 0, 0, 0, 0};
    double tolv = o.tol;
    std::memcpy(&key.val[12], &tolv, sizeof(double));
    int it = 1;
    while (it <= o.maxit && nconv < (unsigned)bt.nsys) {
        const int block = std::min(o.poll - (it - 1) % o.poll, o.maxit - it + 1);
        // full blocks after the first one replay a captured graph (not while per-launch timings are requested)
        const bool use_graph = !o.prof && it > 1 && block == o.poll;
        if ((e = run_iteration_block(use_graph, key, it, block, st, one_iter)) != cudaSuccess) return (int)e;
        it += block;
        e = cudaMemcpyAsync(&nconv, w.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return (int)e;
        timer.collect();
    }
    timer.collect();
    if constexpr (sizeof(T) == 4) {
        if (paired && (e = pair_unpack(w.xp, x, N, bt.nsys, bt.rhs_per_set, st)) != cudaSuccess) return (int)e;
    }
    int err = 0;
    e = cudaMemcpyAsync(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    if (err) rc = LPM_ERR_TIMEOUT;
    return rc;
}

// ----------------------------------------------------------------------------------------- graph cache
namespace {
// Graph cache: key -> (executable graph, last use).  Bounded; when full, the least recently used entry is destroyed
// (a key only recurs while its buffers stay allocated, so old entries are the ones least likely to come back).
constexpr size_t kGraphCap = 256;
struct GraphEntry {
    cudaGraphExec_t exec;
    unsigned long long used;
};
std::mutex g_graph_mu;
std::map<GraphKey, GraphEntry>* g_graphs = new std::map<GraphKey, GraphEntry>();  // never destroyed
unsigned long long g_graph_clock = 0;
long long g_graph_captures = 0, g_graph_flushes = 0;
}  // namespace

void graph_stats(long long* captures, long long* entries, long long* flushes)
{
    std::lock_guard<std::mutex> g(g_graph_mu);
    if (captures) *captures = g_graph_captures;
    if (entries) *entries = (long long)g_graphs->size();
    if (flushes) *flushes = g_graph_flushes;
}

cudaGraphExec_t graph_find(const GraphKey& k)
{
    std::lock_guard<std::mutex> g(g_graph_mu);
    auto it = g_graphs->find(k);
    if (it == g_graphs->end()) return nullptr;
    it->second.used = ++g_graph_clock;
    return it->second.exec;
}

void graph_put(const GraphKey& k, cudaGraphExec_t e)
{
    std::lock_guard<std::mutex> g(g_graph_mu);
    if (g_graphs->size() >= kGraphCap) {  // evict the least recently used graph
        auto lru = g_graphs->begin();
        for (auto it = g_graphs->begin(); it != g_graphs->end(); ++it)
            if (it->second.used < lru->second.used) lru = it;
        cudaGraphExecDestroy(lru->second.exec);
        g_graphs->erase(lru);
        ++g_graph_flushes;
    }
    (*g_graphs)[k] = GraphEntry{e, ++g_graph_clock};
    ++g_graph_captures;
}

cudaStream_t graph_capture_stream()
{
    thread_local cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess)
        streams[dev] = nullptr;
    return streams[dev];
}

template int cg_solve_fused<float>(const Lattice&, const float*, const float*, const Batch&, const float*,
                                   const uint8_t*, const float*, float*, int, const lpm_cg_opts&, void*, size_t, int*,
                                   double*, int*, cudaStream_t);
template int cg_solve_fused<double>(const Lattice&, const double*, const double*, const Batch&, const double*,
                                    const uint8_t*, const double*, double*, int, const lpm_cg_opts&, void*, size_t,
                                    int*, double*, int*, cudaStream_t);

}  // namespace lpm
