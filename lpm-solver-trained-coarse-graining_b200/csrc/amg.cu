// Aggregation-AMG preconditioned CG for the SC operator on full boxes: FP32, on the pair-packed TMA operator.
//
// The preconditioner of timing/t3d/amg3d.py (AMGGeom / AMG3D) with the settings of timing/t3d/problems.py:19
// (aggregates of 3x3x3, dense coarsest level at <= 1000 unknowns, V(1,1) on the finest level, W-cycles below, rho from
// 5 power iterations) as defaults:
//   * geometry (host, once per handle): free particles of each box aggregated in chunks of a sites per axis, the
//     remainder merged into the last chunk (amg3d.py:45-51); level-0 tentative prolongator P = the orthonormalised
//     rigid-body modes of each aggregate.  For box-shaped aggregates the modified Gram-Schmidt of gmg.py:70-142 on the
//     modes of gmg.py:145-162 yields closed forms: translations / sqrt(n) and the centred rotations (-dy, dx, 0),
//     (0, -dz, dy), (dz, 0, -dx), each divided by its norm, d the offset from the aggregate's centre.  P is therefore
//     never stored: kernels evaluate it from a site's position.  The R factors (coarse rigid modes) are closed-form as
//     well; the levels below run the modified Gram-Schmidt itself, on the host.
//   * numeric setup (device, per coefficient set and box): rho(D^-1 K_ff) of the finest level by power iteration
//     (from the first box of the set, reused for the others as timing/t3d/problems.py:126-128 does); the level-1
//     operator P^T K_ff P by probing: K u of P restricted to one colour class of aggregates (27 classes, aggregate
//     index mod 3 per axis) and one rigid mode at a time, restricted back with P^T (aggregates are at least 3 sites
//     wide and the operator reaches 2 sites, so every aggregate meets one aggregate of each colour); below, 6x6
//     diagonal-block inverses, rho by power iteration and Galerkin products Q^T A Q on 27-point 6x6-block stencils
//     (amg3d.py:253-295); the coarsest stencil assembled dense, symmetrised and inverted (blocked Gauss-Jordan, FP64).
//   * cycle (amg3d.py:579-637): finest level x = w M r, t = m (r - K x) by the pair operator's residual epilogue, P^T t,
//     coarse cycle, x += P e, z = x + w m M (r - K x) by its smoother epilogue (which also forms r.z); coarse levels as
//     amg3d._vc / _coarse with nu_c sweeps and gamma cycles.
//   * PCG (amg3d.py:639-668): x0 = 0, stop at |r| <= tol |b| tested every `check` iterations, per-system freezing,
//     iteration blocks replayed as CUDA graphs.
// Power iterations start from a counter-based normal sequence (start_normal) instead of NumPy's generator; rho is an
// estimate either way.  Vectors of the finest level use the pair layout of the operator (kmv_pair.cu); coarse-level
// vectors are (systems of the box, nodes, 6).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "lpm_amg.h"
#include "lpm_cg.h"
#include "lpm_graph.h"
#include "lpm_tma.h"

namespace lpm {

namespace {

constexpr int AMG_MAXL = 9;  // stencil levels (level 1 .. nlev)
constexpr int AMG_MAXBOX = 8;
constexpr int VB = 256;
constexpr int LB = 128;
constexpr int GJ = 32;            // Gauss-Jordan block
constexpr int PCOL = 3;           // colour classes per probing chunk
constexpr int PQ = 6 * PCOL;      // probe systems per set and chunk
constexpr int PNP = PQ / 2;       // probe pairs per set and chunk
constexpr int ST = 972;           // 27 * 36 coefficients per stencil row
// Level operators are symmetric (A_l = P^T K_ff P with K_ff symmetric), so a stencil is stored as its upper half:
// directions d = 13..26 (the diagonal block and the offsets that come later in (z, y, x) order) at index d - 13; the
// block of direction d < 13 at node I is the transpose of the block of direction 26 - d at node I + off(d).
constexpr int STS = 14 * 36;      // stored coefficients per stencil row
constexpr int RS = 8;             // systems per pass of the group kernels

inline int nchunks(int L, int a) { return std::max(1, L / a); }

__host__ __device__ inline void chunk_range(int c, int a, int nch, int L, int& s0, int& w)
{
    s0 = c * a;
    w = c == nch - 1 ? L - s0 : a;
}

__host__ __device__ inline int chunk_of(int p, int a, int nch)
{
    const int c = p / a;
    return c < nch - 1 ? c : nch - 1;
}

// Counter-based normal numbers of the power iterations: splitmix64 finaliser (Steele, Lea, Flood 2014) of the
// element index and level, two uniforms in (0, 1), Box-Muller.
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ inline double start_normal(int level, int64_t e)
{
    const uint64_t k = ((uint64_t)(level + 1) << 56) ^ ((uint64_t)e << 1);
    const double u1 = ((double)(mix64(k) >> 11) + 0.5) * 0x1p-53;
    const double u2 = ((double)(mix64(k | 1ull) >> 11) + 0.5) * 0x1p-53;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// ------------------------------------------------------------------------------------ finest-level aggregates
struct BoxDev {
    int lo[3], L[3], nch[3];
    int n1;          // level-1 nodes (aggregates)
    float* B1;       // (nsb, n1, 6) restricted residual
    const float* E1; // (nsb, n1, 6) coarse correction
};

// Aggregate of a site and the closed-form tentative prolongator there.
struct Agg {
    int I;
    float d[3];
    float isn, i3, i4, i5;
};

__device__ __forceinline__ bool agg_at(const BoxDev& B, int a, int x, int y, int z, Agg& g)
{
    const int p[3] = {x, y, z};
    int c[3];
    float s2[3];
    float n = 1.f;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int rel = p[ax] - B.lo[ax];
        if (rel < 0 || rel >= B.L[ax]) return false;
        const int ci = chunk_of(rel, a, B.nch[ax]);
        int s0, w;
        chunk_range(ci, a, B.nch[ax], B.L[ax], s0, w);
        c[ax] = ci;
        g.d[ax] = (float)(rel - s0) - 0.5f * (float)(w - 1);
        s2[ax] = (float)(w * w - 1) / 12.f;
        n *= (float)w;
    }
    g.I = (c[2] * B.nch[1] + c[1]) * B.nch[0] + c[0];
    g.isn = 1.f / sqrtf(n);
    g.i3 = 1.f / sqrtf(n * (s2[0] + s2[1]));
    g.i4 = 1.f / sqrtf(n * (s2[1] + s2[2]));
    g.i5 = 1.f / sqrtf(n * (s2[0] + s2[2]));
    return true;
}


__device__ __forceinline__ float agg_col(const Agg& g, int c, int a)  // P[a][c]
{
    switch (c) {
    case 0: return a == 0 ? g.isn : 0.f;
    case 1: return a == 1 ? g.isn : 0.f;
    case 2: return a == 2 ? g.isn : 0.f;
    case 3: return a == 0 ? -g.d[1] * g.i3 : (a == 1 ? g.d[0] * g.i3 : 0.f);
    case 4: return a == 1 ? -g.d[2] * g.i4 : (a == 2 ? g.d[1] * g.i4 : 0.f);
    default: return a == 0 ? g.d[2] * g.i5 : (a == 2 ? -g.d[0] * g.i5 : 0.f);
    }
}

__device__ __forceinline__ bool in_box(const int* fb, int x, int y, int z)
{
    return x >= fb[0] && x <= fb[3] && y >= fb[1] && y <= fb[4] && z >= fb[2] && z <= fb[5];
}

// Block-wide deterministic sum of NV per-thread values into part[(v * nrow + row) * nblk + blockIdx.x].
template <int NV>
__device__ __forceinline__ void block_partials(const double (&v)[NV], double* part, int nrow, int row, double* sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const double t = warp_sum(v[q]);
        if (lane == 0) sh[q * 32 + w] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double acc = 0.0;
        for (int k = 0; k < nw; ++k) acc += sh[threadIdx.x * 32 + k];
        part[((int64_t)threadIdx.x * nrow + row) * gridDim.x + blockIdx.x] = acc;
    }
}

// -------------------------------------------------------------------------------------- PCG vector kernels
struct PairGeom {
    int64_t N;
    int nx, ny;
    int nsys, rps, npp;
};

struct PairQ {
    int pr, set, s0, nl;
};

__device__ __forceinline__ PairQ pair_q(const PairGeom& G)
{
    PairQ q;
    q.pr = blockIdx.y;
    q.set = q.pr / G.npp;
    const int jp = q.pr - q.set * G.npp;
    q.s0 = q.set * G.rps + 2 * jp;
    q.nl = min(2, min(G.rps - 2 * jp, G.nsys - q.s0));
    return q;
}

__device__ __forceinline__ void site_xyz(const PairGeom& G, int64_t i, int& x, int& y, int& z)
{
    x = (int)(i % G.nx);
    const int64_t t = i / G.nx;
    y = (int)(t % G.ny);
    z = (int)(t / G.ny);
}

__device__ __forceinline__ void msolve(const float* __restrict__ Ms, int64_t N, int set, int64_t i, const float r[3],
                                       float z[3])
{
    const float* m = Ms + (int64_t)set * 9 * N + i;
    float m9[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) m9[e] = __ldg(m + (int64_t)e * N);
#pragma unroll
    for (int a = 0; a < 3; ++a) z[a] = m9[3 * a] * r[0] + m9[3 * a + 1] * r[1] + m9[3 * a + 2] * r[2];
}

// Last-block machinery of a per-pair reduction: returns true in the block that completes the pair's partials.
__device__ __forceinline__ bool last_of_pair(unsigned* cnt, int pr, bool* flag)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *flag = atomicAdd(cnt + pr, 1u) == (unsigned)(gridDim.x - 1);
    __syncthreads();
    return *flag;
}

__device__ __forceinline__ double part_total(const double* part, int v, int s, int nsys, int nblk)
{
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int b = lane; b < nblk; b += 32) acc += __ldcg(part + ((int64_t)v * nsys + s) * nblk + b);
    return warp_sum(acc);
}

// r = m b (natural -> pair layout), v = w m M r, p = x = 0; b.b, r.r per system; the last block of a pair initialises
// the scalars (as the fused engine's init).
__global__ void __launch_bounds__(VB) k_amg_init(PairGeom G, const float* __restrict__ b, const int* __restrict__ fbox,
                                                 const float* __restrict__ fw, const float* __restrict__ Ms,
                                                 float* __restrict__ r, float* __restrict__ v, float* __restrict__ p,
                                                 float* __restrict__ xp, FcgScalars sc, double* part, unsigned* cnt,
                                                 double tol, int precheck)
{
    __shared__ double sh[4 * 32];
    __shared__ bool last;
    const PairQ q = pair_q(G);
    double vals[4] = {0.0, 0.0, 0.0, 0.0};  // (b.b, r.r) x lanes
    for (int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x; i < G.N; i += (int64_t)gridDim.x * VB) {
        int x, y, z;
        site_xyz(G, i, x, y, z);
        float rv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, vv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        for (int l = 0; l < q.nl; ++l) {
            const int s = q.s0 + l;
            const bool in = in_box(fbox + 6 * s, x, y, z);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float bv = b[((int64_t)s * G.N + i) * 3 + a];
                vals[2 * l] += (double)bv * bv;
                rv[l][a] = in ? bv : 0.f;
                vals[2 * l + 1] += (double)rv[l][a] * rv[l][a];
            }
            if (in) {
                float zz[3];
                msolve(Ms, G.N, q.set, i, rv[l], zz);
                const float w = fw[s];
#pragma unroll
                for (int a = 0; a < 3; ++a) vv[l][a] = w * zz[a];
            }
        }
        const int64_t po = ((int64_t)q.pr * G.N + i) * 6;
        float2* r2 = reinterpret_cast<float2*>(r + po);
        float2* v2 = reinterpret_cast<float2*>(v + po);
        float2* p2 = reinterpret_cast<float2*>(p + po);
        float2* x2 = reinterpret_cast<float2*>(xp + po);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            r2[a] = make_float2(rv[0][a], rv[1][a]);
            v2[a] = make_float2(vv[0][a], vv[1][a]);
            p2[a] = make_float2(0.f, 0.f);
            x2[a] = make_float2(0.f, 0.f);
        }
    }
    {  // partial rows (value, system): value 0 = b.b, 1 = r.r
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double t = warp_sum(vals[k]);
            if (lane == 0) sh[k * 32 + w] = t;
        }
        __syncthreads();
        if (threadIdx.x < 2 * q.nl) {
            const int l = threadIdx.x >> 1, vv = threadIdx.x & 1;
            double acc = 0.0;
            for (int k = 0; k < nw; ++k) acc += sh[threadIdx.x * 32 + k];
            part[((int64_t)vv * G.nsys + q.s0 + l) * gridDim.x + blockIdx.x] = acc;
        }
    }
    if (!last_of_pair(cnt, q.pr, &last)) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int l = w; l < q.nl; l += VB / 32) {
        const int s = q.s0 + l;
        const double bb = part_total(part, 0, s, G.nsys, gridDim.x);
        const double rr = part_total(part, 1, s, G.nsys, gridDim.x);
        if (lane != 0) continue;
        const double bn = sqrt(bb);
        const double rel = bn > 0.0 ? sqrt(rr) / bn : 0.0;
        const bool finite = isfinite(bn) && isfinite(rr);
        int act = bn > 0.0 && finite;
        if (act && precheck && rel <= (sc.tols ? sc.tols[s] : tol)) act = 0;
        sc.bn[s] = bn;
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

// r -= alpha m Ap, r.r; v = w m M r (the first smoothing step of the cycle); the last block of a pair tests
// convergence every `check` iterations and freezes converged systems.  x += alpha p is left to the p-update, which
// reads p anyway (alpha stays set for a system frozen here until the next operator launch zeroes it).
__global__ void __launch_bounds__(VB) k_amg_update(PairGeom G, int it_host, int check, int maxit, double tol,
                                                   const int* __restrict__ fbox, const float* __restrict__ fw,
                                                   const float* __restrict__ Ms, float* __restrict__ r,
                                                   const float* __restrict__ Ap, float* __restrict__ v,
                                                   FcgScalars sc, double* part, unsigned* cnt)
{
    const int it = sc.itp ? *sc.itp : it_host;
    __shared__ double sh[2 * 32];
    __shared__ bool last;
    const PairQ q = pair_q(G);
    const bool on0 = q.nl > 0 && sc.act[q.s0] != 0, on1 = q.nl > 1 && sc.act[q.s0 + 1] != 0;
    const float al0 = on0 ? (float)sc.alpha[q.s0] : 0.f, al1 = on1 ? (float)sc.alpha[q.s0 + 1] : 0.f;
    const float w0 = on0 ? fw[q.s0] : 0.f, w1 = on1 ? fw[q.s0 + 1] : 0.f;
    double rr[2] = {0.0, 0.0};
    // two sites per pass keep twice the loads in flight (67.7 -> 66.2 ms per step of the 16 x 48^3 x 6 batch)
#pragma unroll 2
    for (int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x; i < G.N && (on0 || on1);
         i += (int64_t)gridDim.x * VB) {
        int x, y, z;
        site_xyz(G, i, x, y, z);
        const int64_t po = ((int64_t)q.pr * G.N + i) * 6;
        float2* r2 = reinterpret_cast<float2*>(r + po);
        const float2* a2 = reinterpret_cast<const float2*>(Ap + po);
        float2* v2 = reinterpret_cast<float2*>(v + po);
        float rv[2][3], av[2][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float2 tr = r2[a], ta = a2[a];
            rv[0][a] = tr.x;
            rv[1][a] = tr.y;
            av[0][a] = ta.x;
            av[1][a] = ta.y;
        }
        float vv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            if (!(l ? on1 : on0)) continue;
            const int s = q.s0 + l;
            const bool in = in_box(fbox + 6 * s, x, y, z);
            const float al = l ? al1 : al0;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                rv[l][a] -= in ? al * av[l][a] : 0.f;
                rr[l] += (double)rv[l][a] * rv[l][a];
            }
            if (in) {
                float zz[3];
                msolve(Ms, G.N, q.set, i, rv[l], zz);
                const float w = l ? w1 : w0;
#pragma unroll
                for (int a = 0; a < 3; ++a) vv[l][a] = w * zz[a];
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            r2[a] = make_float2(rv[0][a], rv[1][a]);
            v2[a] = make_float2(vv[0][a], vv[1][a]);
        }
    }
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const double t = warp_sum(rr[l]);
            if (lane == 0) sh[l * 32 + w] = t;
        }
        __syncthreads();
        if (threadIdx.x < q.nl) {
            double acc = 0.0;
            for (int k = 0; k < nw; ++k) acc += sh[threadIdx.x * 32 + k];
            part[(int64_t)(q.s0 + threadIdx.x) * gridDim.x + blockIdx.x] = acc;
        }
    }
    if (!last_of_pair(cnt, q.pr, &last)) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int l = w; l < q.nl; l += VB / 32) {
        const int s = q.s0 + l;
        const double rrn = part_total(part, 0, s, G.nsys, gridDim.x);
        if (lane != 0 || !sc.act[s]) continue;
        sc.rr[s] = rrn;
        const double rel = sqrt(rrn) / sc.bn[s];
        const double tl = sc.tols ? sc.tols[s] : tol;
        if (!isfinite(rrn)) {
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
    if (threadIdx.x == 0) cnt[q.pr] = 0u;
}

// x += alpha p with this iteration's alpha (also for a system frozen by this iteration's update: its alpha is zeroed
// only by the next operator launch), then p = z + beta p for active systems; advances the device iteration counter.
__global__ void __launch_bounds__(VB) k_amg_pupdate(PairGeom G, const float* __restrict__ zb, float* __restrict__ p,
                                                    float* __restrict__ xp, FcgScalars sc)
{
    if (sc.itp && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(sc.itp, 1);
    const PairQ q = pair_q(G);
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= G.N) return;
    const bool on0 = q.nl > 0 && sc.act[q.s0] != 0, on1 = q.nl > 1 && sc.act[q.s0 + 1] != 0;
    const float a0 = q.nl > 0 ? (float)sc.alpha[q.s0] : 0.f, a1 = q.nl > 1 ? (float)sc.alpha[q.s0 + 1] : 0.f;
    const bool mov = a0 != 0.f || a1 != 0.f;
    if (!on0 && !on1 && !mov) return;
    const float b0 = on0 ? (float)sc.beta[q.s0] : 0.f, b1 = on1 ? (float)sc.beta[q.s0 + 1] : 0.f;
    const int64_t po = ((int64_t)q.pr * G.N + i) * 6;
    const float2* z2 = reinterpret_cast<const float2*>(zb + po);
    float2* p2 = reinterpret_cast<float2*>(p + po);
    float2* x2 = reinterpret_cast<float2*>(xp + po);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float2 pp = p2[a];
        if (mov) {
            const float2 xx = x2[a];
            x2[a] = make_float2(xx.x + a0 * pp.x, xx.y + a1 * pp.y);
        }
        if (on0 || on1) {
            const float2 zz = z2[a];
            p2[a] = make_float2(on0 ? zz.x + b0 * pp.x : pp.x, on1 ? zz.y + b1 * pp.y : pp.y);
        }
    }
}

// Finest-level transfers.  A block covers a tile of tw x th aggregates (x, y) of one aggregate layer cz of a box, for
// one pair of systems.  Its work items are (site row r of the aggregates, aggregate): a site row is a contiguous run
// of 24-byte sites (both systems of the pair), and consecutive items take consecutive aggregates of the same row, so
// a warp reads consecutive runs.  Per-item partial sums meet in shared memory and are reduced in a fixed order.
struct TileGeo {
    int cx0, cy0, cz, na, nb, sz, wz, wymax;
};

__host__ __device__ inline TileGeo tile_geo(const int nch[3], const int L[3], int a, int tw, int th, int bx)
{
    TileGeo T;
    const int tiles_x = (nch[0] + tw - 1) / tw, tiles_y = (nch[1] + th - 1) / th;
    const int tx = bx % tiles_x, ty = (bx / tiles_x) % tiles_y;
    T.cz = bx / (tiles_x * tiles_y);
    T.cx0 = tx * tw;
    T.cy0 = ty * th;
    T.na = min(tw, nch[0] - T.cx0);
    T.nb = min(th, nch[1] - T.cy0);
    chunk_range(T.cz, a, nch[2], L[2], T.sz, T.wz);
    int s0, wl;
    chunk_range(T.cy0 + T.nb - 1, a, nch[1], L[1], s0, wl);
    T.wymax = max(wl, T.nb > 1 ? a : wl);
    return T;
}

// tile shape (tw, th) for an aggregate grid nch over extents L, with the shared-memory bytes of one block
struct TileShape {
    int tw, th, tiles;
    size_t smem;
};

inline TileShape tile_shape(const int nch[3], const int L[3], int a, int floats_per_item)
{
    int wy = 0, wz = 0;
    for (int c = 0; c < nch[1]; ++c) {
        int s0, w;
        chunk_range(c, a, nch[1], L[1], s0, w);
        wy = std::max(wy, w);
    }
    for (int c = 0; c < nch[2]; ++c) {
        int s0, w;
        chunk_range(c, a, nch[2], L[2], s0, w);
        wz = std::max(wz, w);
    }
    const int rows = wy * wz;
    const int cap = std::max(1, std::min(32, (48 * 1024) / (rows * floats_per_item * 4)));
    TileShape t;
    t.tw = std::min(nch[0], cap);
    t.th = std::max(1, std::min(nch[1], cap / t.tw));
    t.tiles = (nch[0] + t.tw - 1) / t.tw * ((nch[1] + t.th - 1) / t.th) * nch[2];
    t.smem = (size_t)rows * t.tw * t.th * floats_per_item * 4;
    return t;
}

__device__ __forceinline__ void agg_scales(int wx, int wy, int wz, float& isn, float& i3, float& i4, float& i5)
{
    const float s2x = (float)(wx * wx - 1) / 12.f, s2y = (float)(wy * wy - 1) / 12.f, s2z = (float)(wz * wz - 1) / 12.f;
    const float n = (float)(wx * wy * wz);
    isn = 1.f / sqrtf(n);
    i3 = 1.f / sqrtf(n * (s2x + s2y));
    i4 = 1.f / sqrtf(n * (s2y + s2z));
    i5 = 1.f / sqrtf(n * (s2x + s2z));
}

// Restriction of the probing setup (aggregates wider than k_galerkin0 covers): t is K of probe pair
// pr = set * PNP + jp of chunk `chunk`; writes A1[set][d, :, mode][I] for the colour-class neighbour J = I + off(d) of
// each aggregate I (stored half, d >= 13).  A block covers a tile of tw x th aggregates of one aggregate layer; its
// items (site row, aggregate) read contiguous runs of 24-byte sites and meet in shared memory in a fixed order.
__global__ void __launch_bounds__(256) k_restrict_probe(BoxDev B, int a, int tw, int th, int nx, int ny, int64_t N,
                                                        const float* __restrict__ t, int chunk, float* __restrict__ A1)
{
    extern __shared__ float red[];
    const int pr = blockIdx.y;
    const TileGeo T = tile_geo(B.nch, B.L, a, tw, th, blockIdx.x);
    const int rows = T.wymax * T.wz, nab = T.na * T.nb;
    for (int it = threadIdx.x; it < rows * nab; it += blockDim.x) {
        const int ia = it % T.na, iy = (it / T.na) % T.nb, r = it / nab;
        const int ry = r % T.wymax, rz = r / T.wymax;
        int sx, wx, sy, wy;
        chunk_range(T.cx0 + ia, a, B.nch[0], B.L[0], sx, wx);
        chunk_range(T.cy0 + iy, a, B.nch[1], B.L[1], sy, wy);
        float acc[2][6] = {{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
        if (ry < wy) {
            const float dy = (float)ry - 0.5f * (float)(wy - 1), dz = (float)rz - 0.5f * (float)(T.wz - 1);
            const int y = B.lo[1] + sy + ry, z = B.lo[2] + T.sz + rz;
            const float2* rowp = reinterpret_cast<const float2*>(
                t + ((int64_t)pr * N + ((int64_t)z * ny + y) * nx + B.lo[0] + sx) * 6);
            for (int px = 0; px < wx; ++px) {
                const float dx = (float)px - 0.5f * (float)(wx - 1);
                const float2 v0 = rowp[3 * px], v1 = rowp[3 * px + 1], v2 = rowp[3 * px + 2];
                const float t0[2] = {v0.x, v0.y}, t1[2] = {v1.x, v1.y}, t2[2] = {v2.x, v2.y};
#pragma unroll
                for (int l = 0; l < 2; ++l) {
                    acc[l][0] += t0[l];
                    acc[l][1] += t1[l];
                    acc[l][2] += t2[l];
                    acc[l][3] += dx * t1[l] - dy * t0[l];
                    acc[l][4] += dy * t2[l] - dz * t1[l];
                    acc[l][5] += dz * t0[l] - dx * t2[l];
                }
            }
        }
        float* o = red + (size_t)it * 12;
#pragma unroll
        for (int l = 0; l < 2; ++l)
#pragma unroll
            for (int k = 0; k < 6; ++k) o[l * 6 + k] = acc[l][k];
    }
    __syncthreads();
    for (int o = threadIdx.x; o < nab * 12; o += blockDim.x) {
        const int ab = o / 12, l = (o % 12) / 6, c = o % 6;
        const int ia = ab % T.na, iy = ab / T.na;
        float v = 0.f;
        for (int r = 0; r < rows; ++r) v += red[((size_t)r * nab + ab) * 12 + l * 6 + c];
        int sx, wx, sy, wy;
        chunk_range(T.cx0 + ia, a, B.nch[0], B.L[0], sx, wx);
        chunk_range(T.cy0 + iy, a, B.nch[1], B.L[1], sy, wy);
        float isn, i3, i4, i5;
        agg_scales(wx, wy, T.wz, isn, i3, i4, i5);
        v *= c < 3 ? isn : (c == 3 ? i3 : (c == 4 ? i4 : i5));
        const int cx = T.cx0 + ia, cy = T.cy0 + iy;
        const int I = (T.cz * B.nch[1] + cy) * B.nch[0] + cx;
        const int set = pr / PNP, qq = 2 * (pr % PNP) + l;
        const int colq = chunk * PCOL + qq / 6, mode = qq % 6;
        const int cc[3] = {cx, cy, T.cz}, gcol[3] = {colq % 3, (colq / 3) % 3, colq / 9};
        int off[3];
        bool ok = true;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const int m = ((gcol[ax] - cc[ax]) % 3 + 3) % 3;
            off[ax] = m == 2 ? -1 : m;
            const int J = cc[ax] + off[ax];
            ok = ok && J >= 0 && J < B.nch[ax];
        }
        if (!ok) continue;
        const int d = ((off[2] + 1) * 3 + off[1] + 1) * 3 + off[0] + 1;
        if (d >= 13) A1[((int64_t)set * STS + (d - 13) * 36 + c * 6 + mode) * B.n1 + I] = v;
    }
}

// v += P e1 on the lanes of pair entry (pr, j lane 0, j lane 1) that belong to this box; a lane of another box is never
// written (4-byte stores when only one lane is in the box).  Tiled as k_restrict_probe, one item per site row.
__global__ void __launch_bounds__(256) k_prolong0(BoxDev B, int a, int tw, int th, int nx, int ny, int64_t N,
                                                  const int* __restrict__ pent, const int* __restrict__ sys,
                                                  const int* __restrict__ act, float* __restrict__ v)
{
    const int pr = pent[3 * blockIdx.y], j0 = pent[3 * blockIdx.y + 1], j1 = pent[3 * blockIdx.y + 2];
    const bool on0 = j0 >= 0 && (!act || act[sys[j0]]), on1 = j1 >= 0 && (!act || act[sys[j1]]);
    if (!on0 && !on1) return;
    const TileGeo T = tile_geo(B.nch, B.L, a, tw, th, blockIdx.x);
    const int rows = T.wymax * T.wz, nab = T.na * T.nb;
    for (int it = threadIdx.x; it < rows * nab; it += blockDim.x) {
        const int ia = it % T.na, iy = (it / T.na) % T.nb, r = it / nab;
        const int ry = r % T.wymax, rz = r / T.wymax;
        int sx, wx, sy, wy;
        chunk_range(T.cx0 + ia, a, B.nch[0], B.L[0], sx, wx);
        chunk_range(T.cy0 + iy, a, B.nch[1], B.L[1], sy, wy);
        if (ry >= wy) continue;
        float isn, i3, i4, i5;
        agg_scales(wx, wy, T.wz, isn, i3, i4, i5);
        const int I = (T.cz * B.nch[1] + T.cy0 + iy) * B.nch[0] + T.cx0 + ia;
        float f[2][6];
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const int jj = l ? j1 : j0;
            const bool on = l ? on1 : on0;
            const float* e = B.E1 + ((int64_t)(on ? jj : 0) * B.n1 + I) * 6;
            f[l][0] = on ? isn * e[0] : 0.f;
            f[l][1] = on ? isn * e[1] : 0.f;
            f[l][2] = on ? isn * e[2] : 0.f;
            f[l][3] = on ? i3 * e[3] : 0.f;
            f[l][4] = on ? i4 * e[4] : 0.f;
            f[l][5] = on ? i5 * e[5] : 0.f;
        }
        const float dy = (float)ry - 0.5f * (float)(wy - 1), dz = (float)rz - 0.5f * (float)(T.wz - 1);
        const int y = B.lo[1] + sy + ry, z = B.lo[2] + T.sz + rz;
        float* rowp = v + ((int64_t)pr * N + ((int64_t)z * ny + y) * nx + B.lo[0] + sx) * 6;
        for (int px = 0; px < wx; ++px) {
            const float dx = (float)px - 0.5f * (float)(wx - 1);
            float add[2][3];
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                add[l][0] = f[l][0] - dy * f[l][3] + dz * f[l][5];
                add[l][1] = f[l][1] + dx * f[l][3] - dz * f[l][4];
                add[l][2] = f[l][2] + dy * f[l][4] - dx * f[l][5];
            }
            float2* p2 = reinterpret_cast<float2*>(rowp + 6 * px);
            if (on0 && on1) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float2 o = p2[k];
                    p2[k] = make_float2(o.x + add[0][k], o.y + add[1][k]);
                }
            } else {
                const int l = on1 ? 1 : 0;
#pragma unroll
                for (int k = 0; k < 3; ++k) rowp[6 * px + 2 * k + l] += add[l][k];
            }
        }
    }
}


// Finest-level restriction of the cycle, B1[j][I] = P_I^T t for the lanes of pair entry (pr, j lane 0, j lane 1) in
// this box, one thread per (aggregate I, pair entry): the thread walks I's sites in a fixed order (z, y, x), so its
// sums need no shared memory or barrier and do not depend on scheduling; consecutive threads take x-adjacent
// aggregates, whose site rows are adjacent in memory.  (56 -> 37 us per launch at 16 x 48^3 x 6 against a tiled
// kernel with per-row items.  The same shape for the prolongation measured slower, 69 -> 106 us: each thread's
// read-modify-write chain over its aggregate serialises, so k_prolong0 keeps one item per site row.)
constexpr int TB = 128;
struct AggSpan {
    int sx, wx, sy, wy, sz, wz;
    float isn, i3, i4, i5;
};
__device__ __forceinline__ AggSpan agg_span(const BoxDev& B, int a, int I)
{
    AggSpan s;
    const int cx = I % B.nch[0], cy = (I / B.nch[0]) % B.nch[1], cz = I / (B.nch[0] * B.nch[1]);
    chunk_range(cx, a, B.nch[0], B.L[0], s.sx, s.wx);
    chunk_range(cy, a, B.nch[1], B.L[1], s.sy, s.wy);
    chunk_range(cz, a, B.nch[2], B.L[2], s.sz, s.wz);
    agg_scales(s.wx, s.wy, s.wz, s.isn, s.i3, s.i4, s.i5);
    return s;
}

__global__ void __launch_bounds__(TB) k_restrict_agg(BoxDev B, int a, int nx, int ny, int64_t N,
                                                     const int* __restrict__ pent, const int* __restrict__ sys,
                                                     const int* __restrict__ act, const float* __restrict__ t)
{
    const int I = blockIdx.x * TB + threadIdx.x;
    if (I >= B.n1) return;
    const int pr = pent[3 * blockIdx.y], j0 = pent[3 * blockIdx.y + 1], j1 = pent[3 * blockIdx.y + 2];
    const bool on0 = j0 >= 0 && (!act || act[sys[j0]]), on1 = j1 >= 0 && (!act || act[sys[j1]]);
    if (!on0 && !on1) return;
    const AggSpan s = agg_span(B, a, I);
    float acc[2][6] = {{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
    for (int rz = 0; rz < s.wz; ++rz) {
        const float dz = (float)rz - 0.5f * (float)(s.wz - 1);
        for (int ry = 0; ry < s.wy; ++ry) {
            const float dy = (float)ry - 0.5f * (float)(s.wy - 1);
            const int y = B.lo[1] + s.sy + ry, z = B.lo[2] + s.sz + rz;
            const float2* rowp = reinterpret_cast<const float2*>(
                t + ((int64_t)pr * N + ((int64_t)z * ny + y) * nx + B.lo[0] + s.sx) * 6);
            for (int px = 0; px < s.wx; ++px) {
                const float dx = (float)px - 0.5f * (float)(s.wx - 1);
                const float2 v0 = __ldg(rowp + 3 * px), v1 = __ldg(rowp + 3 * px + 1), v2 = __ldg(rowp + 3 * px + 2);
                const float t0[2] = {v0.x, v0.y}, t1[2] = {v1.x, v1.y}, t2[2] = {v2.x, v2.y};
#pragma unroll
                for (int l = 0; l < 2; ++l) {
                    acc[l][0] += t0[l];
                    acc[l][1] += t1[l];
                    acc[l][2] += t2[l];
                    acc[l][3] += dx * t1[l] - dy * t0[l];
                    acc[l][4] += dy * t2[l] - dz * t1[l];
                    acc[l][5] += dz * t0[l] - dx * t2[l];
                }
            }
        }
    }
    const float sc[6] = {s.isn, s.isn, s.isn, s.i3, s.i4, s.i5};
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        if (!(l ? on1 : on0)) continue;
        float* o = B.B1 + ((int64_t)(l ? j1 : j0) * B.n1 + I) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) o[c] = acc[l][c] * sc[c];
    }
}

// ----------------------------------------------------------------------------------------- probing setup
// Probe systems of one chunk: per set PQ systems q = 6 * colour + mode; value P[:, mode] on the aggregates of the
// colour class (chunk * PCOL + q / 6), zero elsewhere.  Pair layout with PNP pairs per set.
__global__ void __launch_bounds__(VB) k_probe_gen(BoxDev B, int a, int nx, int ny, int64_t N, int chunk,
                                                  float* __restrict__ v)
{
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= N) return;
    const int pr = blockIdx.y, jp = pr % PNP;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((int64_t)nx * ny));
    Agg g;
    const bool in = agg_at(B, a, x, y, z, g);
    if (!in) return;  // zero from the memset before the first chunk
    const int cx = g.I % B.nch[0], cy = (g.I / B.nch[0]) % B.nch[1], cz = g.I / (B.nch[0] * B.nch[1]);
    const int col = (cz % 3) * 9 + (cy % 3) * 3 + cx % 3;
    // the sites of other colour classes hold zero already: write this chunk's classes and clear the previous chunk's
    if (col / PCOL != chunk && col / PCOL != chunk - 1) return;
    float val[2][3];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const int qq = 2 * jp + l;
        const int colq = chunk * PCOL + qq / 6, mode = qq % 6;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) val[l][ax] = (in && col == colq) ? agg_col(g, mode, ax) : 0.f;
    }
    float2* o = reinterpret_cast<float2*>(v + ((int64_t)pr * N + i) * 6);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) o[ax] = make_float2(val[0][ax], val[1][ax]);
}

// ------------------------------------------------------------------------------- direct level-1 Galerkin product
// A1 = P^T K_ff P from the bond coefficients, the product timing/t3d/amg3d.py:151-198 (_galerkin0 on _krow) forms,
// without probe vectors.  One block per (aggregate J, coefficient set) computes the column block J: the fields
// U_m = P_J e_m (mode m of J, zero off J) are rigid on J, so a bond stretch dL_ik = n_k.(U_i - U_q) vanishes unless
// the bond crosses J's surface, and then it is n_k.P_J(i) (i in J) or -n_k.P_J(q) (q in J).  Hence
//   (1) the shell sums S^c, TS^c of the six fields are nonzero only on J +- 1: they go to a shared table;
//   (2) f_p = (K U_m)_p (lin3d.py:126-149: F_pk = 2 Kn dL + (TS_p^c + TS_q^c)/2 + Tv (S_p^c + S_q^c)/2,
//       f_p = sum_k F_pk n_k) is nonzero only on J +- 2; it is formed for the box's sites there;
//   (3) A1[I, J](r, m) = sum_{p in I} P_I(p)[:, r] . f_p[:, m] for the (up to 27) aggregates I next to J.  P_I(p) is
//       affine in the site's offset d from I's centre, so this needs only the moments sum f and sum d f over I's
//       sites, accumulated in FP64 in a fixed order: the result does not depend on scheduling.
// Every (I, J) pair of neighbours is written by exactly one block.  Missing bonds (leaving the lattice) contribute
// nothing, as in the operator; sites off the box have U = 0 but keep their shell sums (K_ff is K restricted to free
// rows and columns, not the operator of a smaller lattice).  Requires aggregates at most GD_WMAX sites wide and at
// least 2 wide where an axis has several (so J +- 2 meets only J's neighbours; the AMG takes a >= 3): a = 3 gives
// widths 3..5.
constexpr int GD_T = 256;
constexpr int GD_WMAX = 5;
constexpr int GD_SW = 28;  // floats per site of the shell-sum table: [c][S 0..5, TS 6..11], padded (float4 phases)

// Slots whose offset along `axis` is `sgn` (-1, 0, +1), as a bit mask over the 18 slots.
__host__ __device__ constexpr unsigned gd_dir(int axis, int sgn)
{
    unsigned m = 0;
    for (int k = 0; k < 18; ++k) {
        const int d = axis == 0 ? sc_dx(k) : axis == 1 ? sc_dy(k) : sc_dz(k);
        if (d == sgn) m |= 1u << k;
    }
    return m;
}

// Slots k of site p whose neighbour p + o_k lies in the box [lo, hi] (inclusive).
__device__ __forceinline__ unsigned gd_range(const int p[3], const int lo[3], const int hi[3])
{
    constexpr unsigned M[3][3] = {{gd_dir(0, -1), gd_dir(0, 0), gd_dir(0, 1)},
                                  {gd_dir(1, -1), gd_dir(1, 0), gd_dir(1, 1)},
                                  {gd_dir(2, -1), gd_dir(2, 0), gd_dir(2, 1)}};
    unsigned m = 0x3FFFFu;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
#pragma unroll
        for (int d = -1; d <= 1; ++d)
            if (p[ax] + d < lo[ax] || p[ax] + d > hi[ax]) m &= ~M[ax][d + 1];
    return m;
}

struct GalJ {
    int lo[3], hi[3];  // J's sites (inclusive)
    float c[3];        // J's centre
    float isn, i3, i4, i5;
};

// dL of slot k for the six fields of J across a bond crossing J's surface; d: offset of the bond's end in J from J's
// centre, s = -w when p is in J (dL = n.P_J(p), n_k = -w o_k) and +w when q is (dL = -n.P_J(q)).
template <int K>
__device__ __forceinline__ void gd_dl(const GalJ& j, float dx, float dy, float dz, float s, float dl[6])
{
    constexpr float ox = (float)sc_dx(K), oy = (float)sc_dy(K), oz = (float)sc_dz(K);
    dl[0] = s * ox * j.isn;
    dl[1] = s * oy * j.isn;
    dl[2] = s * oz * j.isn;
    dl[3] = s * (oy * dx - ox * dy) * j.i3;
    dl[4] = s * (oz * dy - oy * dz) * j.i4;
    dl[5] = s * (ox * dz - oz * dx) * j.i5;
}

template <int K, typename F>
__device__ __forceinline__ void gd_for(F&& f)
{
    if constexpr (K < 18) {
        f(std::integral_constant<int, K>{});
        gd_for<K + 1>(f);
    }
}

// Shared memory of k_galerkin0 for aggregates at most wm sites wide: the shell-sum table on J +- 1 (reused for the
// moments once step 2 is done) and the f table on J +- 2.
__host__ __device__ inline size_t gd_stab_bytes(int wm)
{
    const size_t e1 = (size_t)wm + 2, s = e1 * e1 * e1 * GD_SW * sizeof(float), m = sizeof(double) * 27 * 18 * 4;
    return ((s > m ? s : m) + 15) & ~size_t(15);
}
__host__ __device__ inline size_t gd_smem(int wm)
{
    const size_t e2 = (size_t)wm + 4;
    return gd_stab_bytes(wm) + e2 * e2 * e2 * 18 * sizeof(float);
}

__global__ void __launch_bounds__(GD_T, 3) k_galerkin0(BoxDev B, int a, int wm, int nx, int ny, int nz, int64_t N,
                                                       const float* __restrict__ Kn, const float* __restrict__ Tv,
                                                       float* __restrict__ A1)
{
    extern __shared__ __align__(16) unsigned char gsm[];
    const int E1 = wm + 2, E2 = wm + 4;
    float* stab = reinterpret_cast<float*>(gsm);                       // (E1^3, GD_SW) shell sums on J +- 1
    double* mom = reinterpret_cast<double*>(gsm);                      // (27, 18, 4) moments, after step 2
    float* ftab = reinterpret_cast<float*>(gsm + gd_stab_bytes(wm));  // (E2^3, 18) f_p on J +- 2, [a * 6 + m]

    const int J = blockIdx.x, set = blockIdx.y;
    const int cj[3] = {J % B.nch[0], (J / B.nch[0]) % B.nch[1], J / (B.nch[0] * B.nch[1])};
    GalJ g;
    int wj[3], r1lo[3], r1hi[3];
    for (int ax = 0; ax < 3; ++ax) {
        int s0;
        chunk_range(cj[ax], a, B.nch[ax], B.L[ax], s0, wj[ax]);
        g.lo[ax] = B.lo[ax] + s0;
        g.hi[ax] = g.lo[ax] + wj[ax] - 1;
        g.c[ax] = (float)g.lo[ax] + 0.5f * (float)(wj[ax] - 1);
        r1lo[ax] = g.lo[ax] - 1;
        r1hi[ax] = g.hi[ax] + 1;
    }
    agg_scales(wj[0], wj[1], wj[2], g.isn, g.i3, g.i4, g.i5);
    const int lat_lo[3] = {0, 0, 0}, lat_hi[3] = {nx - 1, ny - 1, nz - 1};
    const float* kn = Kn + (int64_t)set * 18 * N;
    const float* tv = Tv + (int64_t)set * 18 * N;
    const int e1[3] = {wj[0] + 2, wj[1] + 2, wj[2] + 2};
    const int n1 = e1[0] * e1[1] * e1[2];
    const int sy1 = E1, sz1 = E1 * E1;  // table strides (the table's extent is E1 per axis)
    auto tab_at = [&](int l) -> const float4* { return reinterpret_cast<const float4*>(stab + l * GD_SW); };

    // (1) shell sums on J +- 1.  Only bonds crossing J's surface have a stretch: a site of J through its slots leaving
    // J, a site outside through its slots entering J.  Sites off the lattice hold zero.
    for (int t = threadIdx.x; t < n1; t += GD_T) {
        const int lx = t % e1[0], ly = (t / e1[0]) % e1[1], lz = t / (e1[0] * e1[1]);
        const int p3[3] = {r1lo[0] + lx, r1lo[1] + ly, r1lo[2] + lz};
        float s[24];
#pragma unroll
        for (int m = 0; m < 24; ++m) s[m] = 0.f;
        if (p3[0] >= 0 && p3[0] < nx && p3[1] >= 0 && p3[1] < ny && p3[2] >= 0 && p3[2] < nz) {
            const int64_t i = ((int64_t)p3[2] * ny + p3[1]) * nx + p3[0];
            const bool pj = p3[0] >= g.lo[0] && p3[0] <= g.hi[0] && p3[1] >= g.lo[1] && p3[1] <= g.hi[1] &&
                            p3[2] >= g.lo[2] && p3[2] <= g.hi[2];
            const unsigned qj = gd_range(p3, g.lo, g.hi);
            const unsigned cross = gd_range(p3, lat_lo, lat_hi) & (pj ? ~qj : qj);
            const float dx = (float)p3[0] - g.c[0], dy = (float)p3[1] - g.c[1], dz = (float)p3[2] - g.c[2];
            gd_for<0>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                if (!((cross >> k) & 1u)) return;
                constexpr float w = k < 6 ? 1.f : (float)INV_SQRT2;
                constexpr int c = k < 6 ? 0 : 12;
                float dl[6];
                if (pj)
                    gd_dl<k>(g, dx, dy, dz, -w, dl);
                else
                    gd_dl<k>(g, dx + sc_dx(k), dy + sc_dy(k), dz + sc_dz(k), w, dl);
                const float t_ = __ldg(tv + (int64_t)k * N + i);
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    s[c + m] += dl[m];
                    s[c + 6 + m] = fmaf(t_, dl[m], s[c + 6 + m]);
                }
            });
        }
        float4* o = reinterpret_cast<float4*>(stab + ((lz * E1 + ly) * E1 + lx) * GD_SW);
#pragma unroll
        for (int v = 0; v < 6; ++v) o[v] = make_float4(s[4 * v], s[4 * v + 1], s[4 * v + 2], s[4 * v + 3]);
    }
    __syncthreads();

    // (2) f_p on the box's sites of J +- 2.  Items 0..n1-1: the sites of J +- 1 (every slot may contribute); items
    // n1..n1+n2-1: the sites of J +- 2 outside J +- 1, which have no shell sums and no crossing bond, so only their
    // slots reaching into J +- 1 contribute (F = TS_q/2 + Tv S_q/2), one to five of them.
    const int e2[3] = {wj[0] + 4, wj[1] + 4, wj[2] + 4};
    const int n2 = e2[0] * e2[1] * e2[2];
    const int bhi[3] = {B.lo[0] + B.L[0] - 1, B.lo[1] + B.L[1] - 1, B.lo[2] + B.L[2] - 1};
    for (int t = threadIdx.x; t < n1 + n2; t += GD_T) {
        int l2[3];
        if (t < n1) {
            l2[0] = t % e1[0] + 1;
            l2[1] = (t / e1[0]) % e1[1] + 1;
            l2[2] = t / (e1[0] * e1[1]) + 1;
        } else {
            const int u = t - n1;
            l2[0] = u % e2[0];
            l2[1] = (u / e2[0]) % e2[1];
            l2[2] = u / (e2[0] * e2[1]);
            if (l2[0] >= 1 && l2[0] <= e1[0] && l2[1] >= 1 && l2[1] <= e1[1] && l2[2] >= 1 && l2[2] <= e1[2])
                continue;  // a site of J +- 1: item t < n1
        }
        const int p3[3] = {g.lo[0] - 2 + l2[0], g.lo[1] - 2 + l2[1], g.lo[2] - 2 + l2[2]};
        if (p3[0] < B.lo[0] || p3[0] > bhi[0] || p3[1] < B.lo[1] || p3[1] > bhi[1] || p3[2] < B.lo[2] ||
            p3[2] > bhi[2])
            continue;  // no row of K_ff
        const int64_t i = ((int64_t)p3[2] * ny + p3[1]) * nx + p3[0];
        const unsigned valid = gd_range(p3, lat_lo, lat_hi);
        const unsigned qr1 = gd_range(p3, r1lo, r1hi) & valid;
        const int lp = ((l2[2] - 1) * E1 + (l2[1] - 1)) * E1 + (l2[0] - 1);  // table index (p's own: J +- 1 only)
        float f[18];
#pragma unroll
        for (int m = 0; m < 18; ++m) f[m] = 0.f;
        auto add_f = [&](auto kc, const float F[6]) {  // f += F n_k, n_k = -w o_k
            constexpr int k = decltype(kc)::value;
            constexpr float w = k < 6 ? 1.f : (float)INV_SQRT2;
            constexpr int o3[3] = {sc_dx(k), sc_dy(k), sc_dz(k)};
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                if (o3[ax] == 0) continue;
                const float nk = -w * (float)o3[ax];
#pragma unroll
                for (int m = 0; m < 6; ++m) f[ax * 6 + m] = fmaf(nk, F[m], f[ax * 6 + m]);
            }
        };
        auto sums = [&](int l, int c, float sv[12]) {
            const float4* p4 = tab_at(l) + c * 3;
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const float4 q = p4[v];
                sv[4 * v] = q.x;
                sv[4 * v + 1] = q.y;
                sv[4 * v + 2] = q.z;
                sv[4 * v + 3] = q.w;
            }
        };
        if (t < n1) {
            const bool pj = p3[0] >= g.lo[0] && p3[0] <= g.hi[0] && p3[1] >= g.lo[1] && p3[1] <= g.hi[1] &&
                            p3[2] >= g.lo[2] && p3[2] <= g.hi[2];
            const unsigned qj = gd_range(p3, g.lo, g.hi);
            const unsigned cross = valid & (pj ? ~qj : qj);
            const float dx = (float)p3[0] - g.c[0], dy = (float)p3[1] - g.c[1], dz = (float)p3[2] - g.c[2];
            float tvp[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) tvp[k] = __ldg(tv + (int64_t)k * N + i);
            float sp[24];
            sums(lp, 0, sp);
            sums(lp, 1, sp + 12);
            // p's own shell sums enter every slot of their shell: sum_k n_k (TS_p^c + Tv_pk S_p^c) / 2 =
            // (s^c (x) TS_p^c + T^c (x) S_p^c) / 2 with s^c = sum n_k and T^c = sum Tv_pk n_k over the valid slots
            float sv[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}}, tn[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
            gd_for<0>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                if (!((valid >> k) & 1u)) return;
                constexpr int c = k < 6 ? 0 : 1;
                constexpr float w = k < 6 ? 1.f : (float)INV_SQRT2;
                constexpr int o3[3] = {sc_dx(k), sc_dy(k), sc_dz(k)};
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    if (o3[ax] == 0) continue;
                    const float nk = -w * (float)o3[ax];
                    sv[c][ax] += nk;
                    tn[c][ax] = fmaf(tvp[k], nk, tn[c][ax]);
                }
            });
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int ax = 0; ax < 3; ++ax)
#pragma unroll
                    for (int m = 0; m < 6; ++m)
                        f[ax * 6 + m] = fmaf(0.5f * sv[c][ax], sp[12 * c + 6 + m],
                                             fmaf(0.5f * tn[c][ax], sp[12 * c + m], f[ax * 6 + m]));
            // the neighbour's shell sums and the bond stretch, per slot
            gd_for<0>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                const bool qin = (qr1 >> k) & 1u, cr = (cross >> k) & 1u;
                if (!qin && !cr) return;
                constexpr int c = k < 6 ? 0 : 1;
                float F[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (qin) {
                    float sq[12];
                    sums(lp + sc_dx(k) + sc_dy(k) * sy1 + sc_dz(k) * sz1, c, sq);
                    const float tvh = 0.5f * tvp[k];
#pragma unroll
                    for (int m = 0; m < 6; ++m) F[m] = fmaf(tvh, sq[m], 0.5f * sq[6 + m]);
                }
                if (cr) {
                    constexpr float w = k < 6 ? 1.f : (float)INV_SQRT2;
                    float dl[6];
                    if (pj)
                        gd_dl<k>(g, dx, dy, dz, -w, dl);
                    else
                        gd_dl<k>(g, dx + sc_dx(k), dy + sc_dy(k), dz + sc_dz(k), w, dl);
                    const float kn2 = 2.f * __ldg(kn + (int64_t)k * N + i);
#pragma unroll
                    for (int m = 0; m < 6; ++m) F[m] = fmaf(kn2, dl[m], F[m]);
                }
                add_f(kc, F);
            });
        } else if (qr1) {
            gd_for<0>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                if (!((qr1 >> k) & 1u)) return;
                constexpr int c = k < 6 ? 0 : 1;
                float sq[12];
                sums(lp + sc_dx(k) + sc_dy(k) * sy1 + sc_dz(k) * sz1, c, sq);
                const float tvh = 0.5f * __ldg(tv + (int64_t)k * N + i);
                float F[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) F[m] = fmaf(tvh, sq[m], 0.5f * sq[6 + m]);
                add_f(kc, F);
            });
        }
        float* o = ftab + ((l2[2] * E2 + l2[1]) * E2 + l2[0]) * 18;
#pragma unroll
        for (int m = 0; m < 18; ++m) o[m] = f[m];
    }
    __syncthreads();  // the shell-sum table is dead from here: its memory takes the moments

    // (3) moments sum f, sum dx f, sum dy f, sum dz f over the sites of each neighbour I within J +- 2.  Only the
    // stored half is formed: I = J + e - (1, 1, 1) has J in direction d = 26 - e of I, kept when d >= 13 (e <= 13).
    for (int it = threadIdx.x; it < 14 * 18; it += GD_T) {
        const int e = it / 18, am = it % 18;
        const int ci[3] = {cj[0] + e % 3 - 1, cj[1] + (e / 3) % 3 - 1, cj[2] + e / 9 - 1};
        if (ci[0] < 0 || ci[0] >= B.nch[0] || ci[1] < 0 || ci[1] >= B.nch[1] || ci[2] < 0 || ci[2] >= B.nch[2])
            continue;
        int lo[3], hi[3];
        float cc[3];
        for (int ax = 0; ax < 3; ++ax) {
            int s0, w;
            chunk_range(ci[ax], a, B.nch[ax], B.L[ax], s0, w);
            const int il = B.lo[ax] + s0;
            cc[ax] = (float)il + 0.5f * (float)(w - 1);
            lo[ax] = max(il, g.lo[ax] - 2);
            hi[ax] = min(il + w - 1, g.hi[ax] + 2);
        }
        double m0 = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    const int l = ((z - g.lo[2] + 2) * E2 + (y - g.lo[1] + 2)) * E2 + (x - g.lo[0] + 2);
                    const double v = (double)ftab[l * 18 + am];
                    m0 += v;
                    mx += (double)((float)x - cc[0]) * v;
                    my += (double)((float)y - cc[1]) * v;
                    mz += (double)((float)z - cc[2]) * v;
                }
        double* o = mom + (size_t)it * 4;
        o[0] = m0;
        o[1] = mx;
        o[2] = my;
        o[3] = mz;
    }
    __syncthreads();

    // (4) A1[I][d][r][m] with J = I + off(d): off = -e
    const int n1agg = B.n1;
    for (int it = threadIdx.x; it < 14 * 36; it += GD_T) {
        const int e = it / 36, r = (it % 36) / 6, m = it % 6;
        const int ci[3] = {cj[0] + e % 3 - 1, cj[1] + (e / 3) % 3 - 1, cj[2] + e / 9 - 1};
        if (ci[0] < 0 || ci[0] >= B.nch[0] || ci[1] < 0 || ci[1] >= B.nch[1] || ci[2] < 0 || ci[2] >= B.nch[2])
            continue;
        int wi[3];
        for (int ax = 0; ax < 3; ++ax) {
            int s0;
            chunk_range(ci[ax], a, B.nch[ax], B.L[ax], s0, wi[ax]);
        }
        float isn, i3, i4, i5;
        agg_scales(wi[0], wi[1], wi[2], isn, i3, i4, i5);
        auto M = [&](int ax, int q) { return mom[((size_t)e * 18 + ax * 6 + m) * 4 + q]; };  // q: 0 sum, 1..3 d
        double v;
        switch (r) {
        case 0: case 1: case 2: v = (double)isn * M(r, 0); break;
        case 3: v = (double)i3 * (M(1, 1) - M(0, 2)); break;
        case 4: v = (double)i4 * (M(2, 2) - M(1, 3)); break;
        default: v = (double)i5 * (M(0, 3) - M(2, 1)); break;
        }
        const int I = (ci[2] * B.nch[1] + ci[1]) * B.nch[0] + ci[0];
        const int d = ((1 - (e / 9 - 1)) * 3 + (1 - ((e / 3) % 3 - 1))) * 3 + (1 - (e % 3 - 1));
        A1[((int64_t)set * STS + (d - 13) * 36 + r * 6 + m) * n1agg + I] = (float)v;
    }
}



// --------------------------------------------------------------------------------- finest power iteration
// Systems q = set * nb0 + k (k-th box of the set) in the pair layout with rps = nb0.
// x = m M x0 (x0 from start_normal, the same for every system)
__global__ void __launch_bounds__(VB) k_pow0_init(PairGeom G, const int* __restrict__ pbox,
                                                  const float* __restrict__ Ms, float* __restrict__ xv)
{
    const PairQ q = pair_q(G);
    const int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x;
    if (i >= G.N) return;
    int x, y, z;
    site_xyz(G, i, x, y, z);
    float r0[3], zz[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) r0[a] = (float)start_normal(0, i * 3 + a);
    msolve(Ms, G.N, q.set, i, r0, zz);
    float o[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int l = 0; l < q.nl; ++l)
        if (in_box(pbox + 6 * (q.s0 + l), x, y, z))
#pragma unroll
            for (int a = 0; a < 3; ++a) o[l][a] = zz[a];
    float2* o2 = reinterpret_cast<float2*>(xv + ((int64_t)q.pr * G.N + i) * 6);
#pragma unroll
    for (int a = 0; a < 3; ++a) o2[a] = make_float2(o[0][a], o[1][a]);
}

// z = m M m y (y = K x); x.x and z.z per system; x = z.  part rows (value, system): 0 = x.x, 1 = z.z.
__global__ void __launch_bounds__(VB) k_pow0_step(PairGeom G, const int* __restrict__ pbox,
                                                  const float* __restrict__ Ms, float* __restrict__ xv,
                                                  const float* __restrict__ yv, double* part)
{
    __shared__ double sh[4 * 32];
    const PairQ q = pair_q(G);
    double vals[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * VB + threadIdx.x; i < G.N; i += (int64_t)gridDim.x * VB) {
        int x, y, z;
        site_xyz(G, i, x, y, z);
        const int64_t po = ((int64_t)q.pr * G.N + i) * 6;
        float2* x2 = reinterpret_cast<float2*>(xv + po);
        const float2* y2 = reinterpret_cast<const float2*>(yv + po);
        float xo[2][3], yo[2][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float2 tx = x2[a], ty = y2[a];
            xo[0][a] = tx.x;
            xo[1][a] = tx.y;
            yo[0][a] = ty.x;
            yo[1][a] = ty.y;
        }
        float zo[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        for (int l = 0; l < q.nl; ++l) {
#pragma unroll
            for (int a = 0; a < 3; ++a) vals[2 * l] += (double)xo[l][a] * xo[l][a];
            if (!in_box(pbox + 6 * (q.s0 + l), x, y, z)) continue;
            msolve(Ms, G.N, q.set, i, yo[l], zo[l]);
#pragma unroll
            for (int a = 0; a < 3; ++a) vals[2 * l + 1] += (double)zo[l][a] * zo[l][a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) x2[a] = make_float2(zo[0][a], zo[1][a]);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double t = warp_sum(vals[k]);
        if (lane == 0) sh[k * 32 + w] = t;
    }
    __syncthreads();
    if (threadIdx.x < 2 * q.nl) {
        const int l = threadIdx.x >> 1, vv = threadIdx.x & 1;
        double acc = 0.0;
        for (int k = 0; k < nw; ++k) acc += sh[threadIdx.x * 32 + k];
        part[((int64_t)vv * G.nsys + q.s0 + l) * gridDim.x + blockIdx.x] = acc;
    }
}

// rho[q] = sqrt(z.z / x.x) of the last step; one warp per system, partials summed in fixed order.
__global__ void k_pow_finish(int nsys, int nblk, const double* __restrict__ part, double* __restrict__ rho)
{
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= nsys) return;
    const double xx = part_total(part, 0, s, nsys, nblk);
    const double zz = part_total(part, 1, s, nsys, nblk);
    if ((threadIdx.x & 31) == 0) rho[s] = xx > 0.0 ? sqrt(zz / xx) : 0.0;
}

// fw[s] = omega / rho0 of the system's set (and box when rho0_per_box); w[set] = omega / rho of a coarse level.
__global__ void k_fine_weights(int nsys, int rps, int nmask, int nb0, const int* __restrict__ box_of_mask,
                               const double* __restrict__ rho0, double omega, float* __restrict__ fw)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const int set = s / rps;
    const int k = nb0 > 1 ? box_of_mask[s % nmask] : 0;
    const double r = rho0[set * nb0 + k];
    fw[s] = r > 0.0 ? (float)(omega / r) : 0.f;
}

__global__ void k_level_weights(int nset, const double* __restrict__ rho, double omega, float* __restrict__ w)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nset) w[s] = rho[s] > 0.0 ? (float)(omega / rho[s]) : 0.f;
}

// ------------------------------------------------------------------------------------------ coarse levels
// The 6 x 6 block of direction d at node I (J = I + off(d)) of an upper-half stencil, row-major into av.
__device__ __forceinline__ void lv_block(const float* __restrict__ As, int64_t n, int set, int I, int J, int d,
                                         float av[36])
{
    if (d >= 13) {
        const float* p = As + ((int64_t)set * STS + (d - 13) * 36) * n + I;
#pragma unroll
        for (int e = 0; e < 36; ++e) av[e] = __ldg(p + (int64_t)e * n);
    } else {
        const float* p = As + ((int64_t)set * STS + (13 - d) * 36) * n + J;
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = 0; c < 6; ++c) av[r * 6 + c] = __ldg(p + (int64_t)(c * 6 + r) * n);
    }
}

struct LvView {
    int gx, gy, gz, n;
    const float* A;     // (nset, STS, n): upper-half stencil
    const float* Minv;  // (nset, 36, n)
    const float* w;     // (nset)
};

// Rows j of a level kernel: system sys[j] (set = sys[j] / rps, skipped when inactive) or, with sys == nullptr, set j.
__device__ __forceinline__ bool row_set(const int* sys, int rps, const int* act, int j, int& set)
{
    if (!sys) {
        set = j;
        return true;
    }
    const int s = sys[j];
    if (act && !act[s]) return false;
    set = s / rps;
    return true;
}

// MODE 0: y = A x;  1: y = b - A x;  2: y = x + w M (b - A x).  out = y, or out += y when acc.  One thread per node
// and system group g = (set, first row j0, rows cnt) -- the systems of one coefficient set in this box, RS per pass --
// so each stencil row of A (and M) is read once for all of them (splitting a group's systems over threads re-reads
// the rows and measured slower).  Rows of inactive systems are skipped.
template <int MODE>
__global__ void __launch_bounds__(LB) k_lv_op(LvView V, const int* __restrict__ grp, const int* __restrict__ sys,
                                              const int* __restrict__ act, const float* __restrict__ x,
                                              const float* __restrict__ b, float* __restrict__ out, int acc)
{
    const int I = blockIdx.x * LB + threadIdx.x;
    if (I >= V.n) return;
    const int set = grp[3 * blockIdx.y], j0 = grp[3 * blockIdx.y + 1], cnt = grp[3 * blockIdx.y + 2];
    const int i0 = I % V.gx, i1 = (I / V.gx) % V.gy, i2 = I / (V.gx * V.gy);
    for (int c0 = 0; c0 < cnt; c0 += RS) {
        const int nc = min(RS, cnt - c0);
        bool on[RS];
        bool any = false;
#pragma unroll
        for (int r = 0; r < RS; ++r) {
            on[r] = r < nc && (!act || act[sys[j0 + c0 + r]]);
            any |= on[r];
        }
        if (!any) continue;
        float y[RS][6];
#pragma unroll
        for (int r = 0; r < RS; ++r)
#pragma unroll
            for (int k = 0; k < 6; ++k) y[r][k] = 0.f;
#pragma unroll 1
        for (int d = 0; d < 27; ++d) {
            const int q0 = i0 + d % 3 - 1, q1 = i1 + (d / 3) % 3 - 1, q2 = i2 + d / 9 - 1;
            if (q0 < 0 || q0 >= V.gx || q1 < 0 || q1 >= V.gy || q2 < 0 || q2 >= V.gz) continue;
            const int Jn = (q2 * V.gy + q1) * V.gx + q0;
            const int64_t Jo = (int64_t)Jn * 6;
            float av[36];
            lv_block(V.A, V.n, set, I, Jn, d, av);
#pragma unroll
            for (int r = 0; r < RS; ++r) {
                if (!on[r]) continue;
                const float* xs = x + (int64_t)(j0 + c0 + r) * V.n * 6 + Jo;
                float xv[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) xv[k] = xs[k];
#pragma unroll
                for (int rr = 0; rr < 6; ++rr)
#pragma unroll
                    for (int k = 0; k < 6; ++k) y[r][rr] += av[rr * 6 + k] * xv[k];
            }
        }
        float m[36];
        float w = 0.f;
        if constexpr (MODE == 2) {
            const float* M = V.Minv + (int64_t)set * 36 * V.n + I;
#pragma unroll
            for (int e = 0; e < 36; ++e) m[e] = __ldg(M + (int64_t)e * V.n);
            w = V.w[set];
        }
#pragma unroll
        for (int r = 0; r < RS; ++r) {
            if (!on[r]) continue;
            const int64_t o = ((int64_t)(j0 + c0 + r) * V.n + I) * 6;
            float res[6];
            if constexpr (MODE == 0) {
#pragma unroll
                for (int k = 0; k < 6; ++k) res[k] = y[r][k];
            } else {
                float tt[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) tt[k] = b[o + k] - y[r][k];
                if constexpr (MODE == 1) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) res[k] = tt[k];
                } else {
#pragma unroll
                    for (int rr = 0; rr < 6; ++rr) {
                        float zr = 0.f;
#pragma unroll
                        for (int k = 0; k < 6; ++k) zr += m[rr * 6 + k] * tt[k];
                        res[rr] = x[o + rr] + w * zr;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) out[o + k] = acc ? out[o + k] + res[k] : res[k];
        }
    }
}

// x = w M b
__global__ void __launch_bounds__(LB) k_lv_bj(LvView V, const int* __restrict__ sys, int rps,
                                              const int* __restrict__ act, const float* __restrict__ b,
                                              float* __restrict__ x)
{
    const int I = blockIdx.x * LB + threadIdx.x;
    const int j = blockIdx.y;
    int set;
    if (I >= V.n || !row_set(sys, rps, act, j, set)) return;
    const int64_t o = ((int64_t)j * V.n + I) * 6;
    const float* M = V.Minv + (int64_t)set * 36 * V.n + I;
    const float w = V.w[set];
    float bv[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) bv[c] = b[o + c];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        float zr = 0.f;
#pragma unroll
        for (int c = 0; c < 6; ++c) zr += __ldg(M + (int64_t)(r * 6 + c) * V.n) * bv[c];
        x[o + r] = w * zr;
    }
}


// x[j][m] += Q_m e[j][agg(m)]   (amg3d.py:313-326)
__global__ void __launch_bounds__(LB) k_lv_prolong(int gx, int gy, int gz, int cx, int cy, int cz, int a,
                                                   const float* __restrict__ Q, const int* __restrict__ sys, int rps,
                                                   const int* __restrict__ act, const float* __restrict__ e,
                                                   float* __restrict__ x)
{
    const int m = blockIdx.x * LB + threadIdx.x;
    const int j = blockIdx.y;
    int set;
    const int n = gx * gy * gz, nc = cx * cy * cz;
    if (m >= n || !row_set(sys, rps, act, j, set)) return;
    const int J = (chunk_of(m / (gx * gy), a, cz) * cy + chunk_of((m / gx) % gy, a, cy)) * cx + chunk_of(m % gx, a, cx);
    const float* ev = e + ((int64_t)j * nc + J) * 6;
    const float* q = Q + (int64_t)m * 36;
    float eg[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) eg[k] = ev[k];
    float* xo = x + ((int64_t)j * n + m) * 6;
#pragma unroll
    for (int a2 = 0; a2 < 6; ++a2) {
        float s = 0.f;
#pragma unroll
        for (int cc = 0; cc < 6; ++cc) s += q[a2 * 6 + cc] * eg[cc];
        xo[a2] += s;
    }
}

// bc[j][J] = sum over the nodes m of coarse node J of Q_m^T r[j][m]   (amg3d.py:298-310), for system j, tiled as the
// finest-level restriction: items are runs of consecutive fine nodes (24 bytes of r and 144 bytes of Q per node).
__global__ void __launch_bounds__(256) k_lv_restrict(int gx, int gy, int gz, int n, int cx, int cy, int cz, int a,
                                                     int tw, int th, const float* __restrict__ Q,
                                                     const int* __restrict__ sys, const int* __restrict__ act,
                                                     const float* __restrict__ r, float* __restrict__ bc)
{
    extern __shared__ float red[];
    const int j = blockIdx.y;
    if (act && !act[sys[j]]) return;
    const int nch[3] = {cx, cy, cz}, L[3] = {gx, gy, gz};
    const TileGeo T = tile_geo(nch, L, a, tw, th, blockIdx.x);
    const int rows = T.wymax * T.wz, nab = T.na * T.nb;
    for (int it = threadIdx.x; it < rows * nab; it += blockDim.x) {
        const int ia = it % T.na, iy = (it / T.na) % T.nb, rr = it / nab;
        const int ry = rr % T.wymax, rz = rr / T.wymax;
        int sx, wx, sy, wy;
        chunk_range(T.cx0 + ia, a, cx, gx, sx, wx);
        chunk_range(T.cy0 + iy, a, cy, gy, sy, wy);
        float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (ry < wy) {
            const int m0 = ((T.sz + rz) * gy + sy + ry) * gx + sx;
            for (int px = 0; px < wx; ++px) {
                const float* rv = r + ((int64_t)j * n + m0 + px) * 6;
                const float* q = Q + (int64_t)(m0 + px) * 36;
                float rl[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) rl[k] = rv[k];
#pragma unroll
                for (int k = 0; k < 6; ++k)
#pragma unroll
                    for (int c = 0; c < 6; ++c) acc[c] += q[k * 6 + c] * rl[k];
            }
        }
        float* o = red + (size_t)it * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) o[c] = acc[c];
    }
    __syncthreads();
    for (int o = threadIdx.x; o < nab * 6; o += blockDim.x) {
        const int ab = o / 6, c = o % 6;
        const int ia = ab % T.na, iy = ab / T.na;
        float v = 0.f;
        for (int rr = 0; rr < rows; ++rr) v += red[((size_t)rr * nab + ab) * 6 + c];
        bc[((int64_t)j * cx * cy * cz + (T.cz * cy + T.cy0 + iy) * cx + T.cx0 + ia) * 6 + c] = v;
    }
}

// out[j] (+)= Ainv[set] rhs[j] on the dense coarsest level (FP32 inverse, rows padded to ncp): a block per (32 rows,
// system group); the group's right-hand sides pass through shared memory in column chunks, each warp owns 4 rows and
// reads them as float4.
constexpr int DR = 32, DC = 512;
__global__ void __launch_bounds__(256) k_dense_apply(int nc, int ncp, const float* __restrict__ Ainv,
                                                     const int* __restrict__ grp, const int* __restrict__ sys,
                                                     const int* __restrict__ act, const float* __restrict__ rhs,
                                                     float* __restrict__ out, int acc)
{
    __shared__ __align__(16) float sr[RS][DC];
    const int set = grp[3 * blockIdx.y], j0 = grp[3 * blockIdx.y + 1], cnt = grp[3 * blockIdx.y + 2];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * DR + w * 4;
    const float* Ab = Ainv + (int64_t)set * ncp * ncp;
    for (int c0 = 0; c0 < cnt; c0 += RS) {
        const int nr = min(RS, cnt - c0);
        bool on[RS];
        bool any = false;
#pragma unroll
        for (int r = 0; r < RS; ++r) {
            on[r] = r < nr && (!act || act[sys[j0 + c0 + r]]);
            any |= on[r];
        }
        if (!any) continue;
        float sa[4][RS];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < RS; ++r) sa[q][r] = 0.f;
        for (int k0 = 0; k0 < ncp; k0 += DC) {
            const int kn = min(DC, ncp - k0);
            __syncthreads();
            for (int e = threadIdx.x; e < RS * DC; e += blockDim.x) {
                const int r = e / DC, k = e % DC;
                sr[r][k] = (r < nr && k < kn && k0 + k < nc && on[r]) ? rhs[(int64_t)(j0 + c0 + r) * nc + k0 + k] : 0.f;
            }
            __syncthreads();
            for (int k4 = lane; 4 * k4 < kn; k4 += 32) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (r0 + q >= nc) continue;
                    const float4 av = *reinterpret_cast<const float4*>(Ab + (int64_t)(r0 + q) * ncp + k0 + 4 * k4);
#pragma unroll
                    for (int r = 0; r < RS; ++r) {
                        const float4 xv = *reinterpret_cast<const float4*>(&sr[r][4 * k4]);
                        sa[q][r] += av.x * xv.x + av.y * xv.y + av.z * xv.z + av.w * xv.w;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < RS; ++r) {
                float v = sa[q][r];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0 && on[r] && r0 + q < nc) {
                    float* po = out + (int64_t)(j0 + c0 + r) * nc + r0 + q;
                    *po = acc ? *po + v : v;
                }
            }
    }
}

// ------------------------------------------------------------------------------------ coarse-level setup
// Minv[set][:, I] = inverse of the diagonal block A[set][13][:, :, I] (Gauss-Jordan in FP64, partial pivoting).
__global__ void k_lv_diag_inv(int n, int nset, const float* __restrict__ A, float* __restrict__ Minv)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int set = blockIdx.y;
    if (I >= n || set >= nset) return;
    double m[6][12];
    const float* Ab = A + (int64_t)set * STS * n + I;  // direction 13, stored first
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            m[r][c] = (double)Ab[(int64_t)(r * 6 + c) * n];
            m[r][6 + c] = r == c ? 1.0 : 0.0;
        }
    for (int k = 0; k < 6; ++k) {
        int pv = k;
        for (int r = k + 1; r < 6; ++r)
            if (fabs(m[r][k]) > fabs(m[pv][k])) pv = r;
        if (pv != k)
            for (int c = 0; c < 12; ++c) {
                const double t = m[k][c];
                m[k][c] = m[pv][c];
                m[pv][c] = t;
            }
        const double ip = m[k][k] != 0.0 ? 1.0 / m[k][k] : 0.0;
        for (int c = 0; c < 12; ++c) m[k][c] *= ip;
        for (int r = 0; r < 6; ++r) {
            if (r == k) continue;
            const double f = m[r][k];
            for (int c = 0; c < 12; ++c) m[r][c] -= f * m[k][c];
        }
    }
    float* Mo = Minv + (int64_t)set * 36 * n + I;
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) Mo[(int64_t)(r * 6 + c) * n] = (float)m[r][6 + c];
}

// x[set] = Minv[set] x0, x0 from start_normal(level, .)
__global__ void k_pow_lv_init(int n, int level, const float* __restrict__ Minv, float* __restrict__ x)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int set = blockIdx.y;
    if (I >= n) return;
    float r0[6];
    for (int c = 0; c < 6; ++c) r0[c] = (float)start_normal(level, (int64_t)I * 6 + c);
    const float* M = Minv + (int64_t)set * 36 * n + I;
    float* o = x + ((int64_t)set * n + I) * 6;
    for (int r = 0; r < 6; ++r) {
        float s = 0.f;
        for (int c = 0; c < 6; ++c) s += M[(int64_t)(r * 6 + c) * n] * r0[c];
        o[r] = s;
    }
}

// z = Minv y; x.x and z.z per set; x = z.
__global__ void __launch_bounds__(LB) k_pow_lv_step(int n, const float* __restrict__ Minv, float* __restrict__ x,
                                                    const float* __restrict__ y, double* part)
{
    __shared__ double sh[2 * 32];
    const int set = blockIdx.y;
    double v[2] = {0.0, 0.0};
    for (int I = blockIdx.x * LB + threadIdx.x; I < n; I += gridDim.x * LB) {
        const int64_t o = ((int64_t)set * n + I) * 6;
        const float* M = Minv + (int64_t)set * 36 * n + I;
        float yv[6];
        for (int c = 0; c < 6; ++c) {
            yv[c] = y[o + c];
            v[0] += (double)x[o + c] * x[o + c];
        }
        for (int r = 0; r < 6; ++r) {
            float s = 0.f;
            for (int c = 0; c < 6; ++c) s += M[(int64_t)(r * 6 + c) * n] * yv[c];
            v[1] += (double)s * s;
            x[o + r] = s;
        }
    }
    block_partials<2>(v, part, gridDim.y, set, sh);
}

// Ac[set][dd][:, :, J] = sum over nodes m of J and stencil offsets d of Q_m^T A[set][d][m] Q_{m+d}
// (amg3d.py:253-295); one block per (coarse node, set), FP32 products accumulated in FP64 in shared memory.
__global__ void __launch_bounds__(256) k_galerkin(int gx, int gy, int gz, int cx, int cy, int cz, int a,
                                                  const float* __restrict__ A, const float* __restrict__ Q,
                                                  float* __restrict__ Ac)
{
    __shared__ double acc[STS];  // the stored half: coarse directions dd = 13..26
    const int J = blockIdx.x, set = blockIdx.y;
    const int n = gx * gy * gz, nc = cx * cy * cz;
    for (int e = threadIdx.x; e < STS; e += blockDim.x) acc[e] = 0.0;
    __syncthreads();
    const int c[3] = {J % cx, (J / cx) % cy, J / (cx * cy)};
    const int g[3] = {gx, gy, gz}, nch[3] = {cx, cy, cz};
    int s0[3], w[3];
    for (int ax = 0; ax < 3; ++ax) chunk_range(c[ax], a, nch[ax], g[ax], s0[ax], w[ax]);
    const int nmem = w[0] * w[1] * w[2];
    for (int item = threadIdx.x; item < nmem * 27; item += blockDim.x) {
        const int mi = item / 27, d = item % 27;
        const int mx = s0[0] + mi % w[0], my = s0[1] + (mi / w[0]) % w[1], mz = s0[2] + mi / (w[0] * w[1]);
        const int nxq = mx + d % 3 - 1, nyq = my + (d / 3) % 3 - 1, nzq = mz + d / 9 - 1;
        if (nxq < 0 || nxq >= gx || nyq < 0 || nyq >= gy || nzq < 0 || nzq >= gz) continue;
        const int m = (mz * gy + my) * gx + mx, q = (nzq * gy + nyq) * gx + nxq;
        const int Jx = chunk_of(nxq, a, cx), Jy = chunk_of(nyq, a, cy), Jz = chunk_of(nzq, a, cz);
        const int dd = ((Jz - c[2] + 1) * 3 + Jy - c[1] + 1) * 3 + Jx - c[0] + 1;
        if (dd < 13) continue;
        float Ab[36], Cq[36];
        lv_block(A, n, set, m, q, d, Ab);
        const float* Qm = Q + (int64_t)m * 36;
        const float* Qq = Q + (int64_t)q * 36;
#pragma unroll
        for (int r = 0; r < 6; ++r)  // C = A Q_q
#pragma unroll
            for (int cc = 0; cc < 6; ++cc) {
                float s = 0.f;
#pragma unroll
                for (int b = 0; b < 6; ++b) s += Ab[r * 6 + b] * __ldg(Qq + b * 6 + cc);
                Cq[r * 6 + cc] = s;
            }
        // Q_m^T C in FP32, accumulated over the members and offsets in FP64
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int cc = 0; cc < 6; ++cc) {
                float s = 0.f;
#pragma unroll
                for (int b = 0; b < 6; ++b) s += __ldg(Qm + b * 6 + r) * Cq[b * 6 + cc];
                atomicAdd(&acc[(dd - 13) * 36 + r * 6 + cc], (double)s);
            }
    }
    __syncthreads();
    float* o = Ac + (int64_t)set * STS * nc + J;
    for (int e = threadIdx.x; e < STS; e += blockDim.x) o[(int64_t)e * nc] = (float)acc[e];
}

// Dense (ncp x ncp) matrix of the coarsest stencil (padding rows / columns: identity).
__global__ void k_dense_build(int gx, int gy, int gz, int ncp, const float* __restrict__ A, double* __restrict__ D)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int d = blockIdx.y, set = blockIdx.z;
    const int n = gx * gy * gz;
    double* Ds = D + (int64_t)set * ncp * ncp;
    if (d == 0 && I < ncp - 6 * n) {
        const int p = 6 * n + I;
        Ds[(int64_t)p * ncp + p] = 1.0;
    }
    if (I >= n) return;
    const int i0 = I % gx, i1 = (I / gx) % gy, i2 = I / (gx * gy);
    const int j0 = i0 + d % 3 - 1, j1 = i1 + (d / 3) % 3 - 1, j2 = i2 + d / 9 - 1;
    if (j0 < 0 || j0 >= gx || j1 < 0 || j1 >= gy || j2 < 0 || j2 >= gz) return;
    const int J = (j2 * gy + j1) * gx + j0;
    float av[36];
    lv_block(A, n, set, I, J, d, av);
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) Ds[(int64_t)(6 * I + r) * ncp + 6 * J + c] = (double)av[r * 6 + c];
}

// D = (D + D^T) / 2 over the leading nc x nc block (as amg3d.py:568-569)
__global__ void k_dense_sym(int nc, int ncp, double* __restrict__ D)
{
    const int i = blockIdx.y * 16 + threadIdx.y, j = blockIdx.x * 16 + threadIdx.x;
    if (i >= nc || j >= nc || j <= i) return;
    double* Ds = D + (int64_t)blockIdx.z * ncp * ncp;
    const double m = 0.5 * (Ds[(int64_t)i * ncp + j] + Ds[(int64_t)j * ncp + i]);
    Ds[(int64_t)i * ncp + j] = m;
    Ds[(int64_t)j * ncp + i] = m;
}

// Blocked in-place Gauss-Jordan inversion of an SPD matrix, block column K:
//   Pinv = inv(D_KK);  D_KJ = Pinv D_KJ;  D_IJ -= D_IK D_KJ;  D_IK = -D_IK Pinv;  D_KK = Pinv   (I, J != K)
__global__ void __launch_bounds__(GJ* GJ) k_gj_diag(int K, int ncp, const double* __restrict__ D,
                                                    double* __restrict__ Pinv)
{
    __shared__ double m[GJ][GJ + 1];
    const int tx = threadIdx.x, ty = threadIdx.y, set = blockIdx.x;
    const double* Ds = D + (int64_t)set * ncp * ncp;
    m[ty][tx] = Ds[(int64_t)(K * GJ + ty) * ncp + K * GJ + tx];
    __syncthreads();
    for (int k = 0; k < GJ; ++k) {
        const double p = m[k][k], rk = m[k][tx], ci = m[ty][k], a = m[ty][tx];
        __syncthreads();
        const double ip = 1.0 / p;
        double v;
        if (ty == k)
            v = tx == k ? ip : rk * ip;
        else
            v = tx == k ? -ci * ip : a - ci * rk * ip;
        m[ty][tx] = v;
        __syncthreads();
    }
    Pinv[((int64_t)set * GJ + ty) * GJ + tx] = m[ty][tx];
}

// Row step: D_KJ = Pinv D_KJ for every block column J != K.  One block per (J, set): the 32 x 32 block and Pinv in
// shared memory, 4 outputs per thread.
__global__ void __launch_bounds__(256) k_gj_row(int K, int ncp, double* __restrict__ D, const double* __restrict__ Pinv)
{
    __shared__ double P[GJ][GJ + 1], X[GJ][GJ + 1];
    const int J = blockIdx.x, set = blockIdx.y;
    if (J == K) return;
    double* Ds = D + (int64_t)set * ncp * ncp;
    const int tx = threadIdx.x % GJ, ty = threadIdx.x / GJ;  // 32 x 8
    for (int r = ty; r < GJ; r += 8) {
        P[r][tx] = Pinv[((int64_t)set * GJ + r) * GJ + tx];
        X[r][tx] = Ds[(int64_t)(K * GJ + r) * ncp + J * GJ + tx];
    }
    __syncthreads();
    for (int r = ty; r < GJ; r += 8) {
        double s = 0.0;
#pragma unroll 8
        for (int k = 0; k < GJ; ++k) s = fma(P[r][k], X[k][tx], s);
        Ds[(int64_t)(K * GJ + r) * ncp + J * GJ + tx] = s;
    }
}

// Trailing step: D_IJ -= D_IK D_KJ for I, J != K, on 64 x 64 tiles (4 x 4 outputs per thread from shared-memory
// panels of D_IK and D_KJ).  A tile may hold part of the pivot row or column block, which it leaves alone.
constexpr int GT = 64;
__global__ void __launch_bounds__(256) k_gj_trail(int K, int ncp, double* __restrict__ D)
{
    __shared__ double Aik[GJ][GT + 1], Akj[GJ][GT];
    const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT, set = blockIdx.z, k0 = K * GJ;
    if (i0 >= ncp || j0 >= ncp) return;
    if ((i0 / GJ == K && i0 + GJ >= ncp) || (j0 / GJ == K && j0 + GJ >= ncp)) return;  // only pivot rows / columns
    double* Ds = D + (int64_t)set * ncp * ncp;
    const int tid = threadIdx.x;
    for (int e = tid; e < GT * GJ; e += 256) {
        const int r = e / GJ, k = e % GJ;
        Aik[k][r] = i0 + r < ncp ? Ds[(int64_t)(i0 + r) * ncp + k0 + k] : 0.0;
        const int kk = e / GT, c = e % GT;
        Akj[kk][c] = j0 + c < ncp ? Ds[(int64_t)(k0 + kk) * ncp + j0 + c] : 0.0;
    }
    __syncthreads();
    const int tr = tid / 16, tc = tid % 16;  // rows tr + 16 q, columns tc + 16 s
    double acc[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int t = 0; t < 4; ++t) acc[q][t] = 0.0;
#pragma unroll 4
    for (int k = 0; k < GJ; ++k) {
        double av[4], bv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            av[q] = Aik[k][tr + 16 * q];
            bv[q] = Akj[k][tc + 16 * q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int t = 0; t < 4; ++t) acc[q][t] = fma(av[q], bv[t], acc[q][t]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int i = i0 + tr + 16 * q;
        if (i >= ncp || i / GJ == K) continue;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int j = j0 + tc + 16 * t;
            if (j < ncp && j / GJ != K) Ds[(int64_t)i * ncp + j] -= acc[q][t];
        }
    }
}

// Column step: D_IK = -D_IK Pinv for every block row I != K, and D_KK = Pinv.  One block per (I, set).
__global__ void __launch_bounds__(256) k_gj_col(int K, int ncp, double* __restrict__ D, const double* __restrict__ Pinv)
{
    __shared__ double P[GJ][GJ + 1], X[GJ][GJ + 1];
    const int I = blockIdx.x, set = blockIdx.y;
    double* Ds = D + (int64_t)set * ncp * ncp;
    const int tx = threadIdx.x % GJ, ty = threadIdx.x / GJ;
    for (int r = ty; r < GJ; r += 8) {
        P[r][tx] = Pinv[((int64_t)set * GJ + r) * GJ + tx];
        X[r][tx] = Ds[(int64_t)(I * GJ + r) * ncp + K * GJ + tx];
    }
    __syncthreads();
    for (int r = ty; r < GJ; r += 8) {
        double s;
        if (I == K) {
            s = P[r][tx];
        } else {
            s = 0.0;
#pragma unroll 8
            for (int k = 0; k < GJ; ++k) s = fma(X[r][k], P[k][tx], s);
            s = -s;
        }
        Ds[(int64_t)(I * GJ + r) * ncp + K * GJ + tx] = s;
    }
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

__global__ void k_repack_ms(const float* __restrict__ M, float* __restrict__ Ms, int64_t N)
{
    const int c = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
#pragma unroll
    for (int e = 0; e < 9; ++e) Ms[((int64_t)c * 9 + e) * N + i] = M[((int64_t)c * N + i) * 9 + e];
}


// -------------------------------------------------------------------------------------------- host geometry
// Modified Gram-Schmidt of a k x 6 block (gmg.py:70-142 on one aggregate): Q (k x 6), R (6 x 6); false when a column
// falls below tol times the largest column norm (rank deficiency).
bool mgs6(const std::vector<double>& blk, int k, double* Q, double* R, double tol)
{
    double scale = 0.0;
    for (int c = 0; c < 6; ++c) {
        double s = 0.0;
        for (int q = 0; q < k; ++q) s += blk[q * 6 + c] * blk[q * 6 + c];
        scale = std::max(scale, std::sqrt(s));
    }
    std::fill(R, R + 36, 0.0);
    std::vector<double> v(k);
    for (int c = 0; c < 6; ++c) {
        for (int q = 0; q < k; ++q) v[q] = blk[q * 6 + c];
        for (int d = 0; d < c; ++d) {
            double pr = 0.0;
            for (int q = 0; q < k; ++q) pr += Q[q * 6 + d] * v[q];
            R[d * 6 + c] = pr;
            for (int q = 0; q < k; ++q) v[q] -= pr * Q[q * 6 + d];
        }
        double nrm = 0.0;
        for (int q = 0; q < k; ++q) nrm += v[q] * v[q];
        nrm = std::sqrt(nrm);
        if (!(nrm > tol * scale && nrm > 0.0)) return false;
        R[c * 6 + c] = nrm;
        for (int q = 0; q < k; ++q) Q[q * 6 + c] = v[q] / nrm;
    }
    return true;
}

}  // namespace
}  // namespace lpm

// ============================================================================================== the handle
struct lpm_amg {
    struct Level {
        int g[3] = {0, 0, 0};
        int n = 0;
        lpm::TileShape tr{};  // tiles of the restriction to the next level
        float *A = nullptr, *Minv = nullptr, *Q = nullptr, *w = nullptr;
        double* rho = nullptr;
        float *B = nullptr, *E = nullptr, *RB = nullptr, *X = nullptr, *X2 = nullptr, *T = nullptr;
        std::vector<double> Qh;  // host copy of the transfer to the next level (n x 36)
    };
    struct Box {
        int lo[3], hi[3], L[3], nch[3];
        int nlev = 0;
        Level lev[lpm::AMG_MAXL];
        int nc = 0, ncp = 0;
        double* Ainv = nullptr;
        int nsb = 0;
        int* sys = nullptr;
        std::vector<int> sys_h;
        int ngrp = 0, npent = 0;
        lpm::TileShape t0{};        // tiles of the finest-level transfers
        float* Ainv32 = nullptr;    // FP32 copy of the dense inverse, applied in the cycle
        int *grp = nullptr, *pent = nullptr;  // system groups (set, j0, cnt); pair entries (pr, j lane 0, j lane 1)
        std::vector<int> grp_h, pent_h;
    };
    lpm::Lattice L{};
    int nsys = 0, rps = 0, nmask = 0, nset = 0, npp = 0, npair = 0, nbox = 0, nb0 = 1;
    lpm_amg_opts o{};
    int dev = 0;
    unsigned long long id = 0, gen = 0;
    std::vector<Box> box;
    std::vector<int> box_of_mask_h;
    int *box_of_mask = nullptr, *fbox = nullptr, *pbox = nullptr, *pgrp = nullptr;
    float* fw = nullptr;
    float *Ms = nullptr, *xp = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr, *v = nullptr;
    lpm::FcgScalars sc{};
    double *vpart = nullptr, *mpart = nullptr, *ppart = nullptr, *rho0 = nullptr, *Pinv = nullptr;
    unsigned *vcnt = nullptr, *mcnt = nullptr;
    int* err = nullptr;
    float *pw_x = nullptr, *pw_y = nullptr;
    int *it_scr = nullptr, *st_scr = nullptr;
    double* rel_scr = nullptr;
    const float *Kn = nullptr, *Tv = nullptr;  // the handle's own copy of the packed FP32 coefficients
    float *Kn_own = nullptr, *Tv_own = nullptr;
    int zchunk = 1, variant = 0, zchunk_probe = 1, zchunk_pow = 1;
    int nblk_pow = 1;
    void* mem = nullptr;
    size_t bytes = 0;
    bool ready = false;
    // the coarse cycles of different boxes run on their own streams (forked from and joined to the caller's)
    std::vector<cudaStream_t> bst;
    std::vector<cudaEvent_t> bev;  // [0]: fork, [1 + k]: join of box k
    ~lpm_amg()
    {
        for (auto s : bst) cudaStreamDestroy(s);
        for (auto e : bev) cudaEventDestroy(e);
        if (mem) cudaFree(mem);
    }
};

namespace lpm {
namespace {

std::atomic<unsigned long long> g_amg_ids{1};

struct Carver2 {
    char* base;
    size_t off;
    template <typename X>
    X* take(size_t n)
    {
        X* q = base ? reinterpret_cast<X*>(base + off) : nullptr;
        off = (off + n * sizeof(X) + 255) & ~size_t(255);
        return q;
    }
};

int pow_blocks(int64_t N) { return (int)std::max<int64_t>(1, std::min<int64_t>((N + VB - 1) / VB, 64)); }

// Carve every device array of the handle (base == nullptr: sizing pass).
void carve_amg(lpm_amg& h, Carver2& c)
{
    const int64_t N = h.L.N;
    h.box_of_mask = c.take<int>(h.nmask);
    h.fbox = c.take<int>((size_t)6 * h.nsys);
    h.pbox = c.take<int>((size_t)6 * h.nset * h.nb0);
    h.pgrp = c.take<int>((size_t)3 * h.nset);
    h.fw = c.take<float>(h.nsys);
    h.Ms = c.take<float>((size_t)h.nset * 9 * N);
    h.Kn_own = c.take<float>((size_t)h.nset * 18 * N);
    h.Tv_own = c.take<float>((size_t)h.nset * 18 * N);
    // finest-level vectors; the probing and power-iteration setup reuses the same memory
    const size_t pv = (size_t)N * 6;
    const size_t solve = (size_t)5 * h.npair * pv;
    const size_t probe = (size_t)2 * h.nset * PNP * pv;
    const size_t powr = (size_t)2 * h.nset * ((h.nb0 + 1) / 2) * pv;
    float* fv = c.take<float>(std::max(solve, std::max(probe, powr)));
    if (fv) {
        h.xp = fv;
        h.r = fv + h.npair * pv;
        h.p = fv + 2 * h.npair * pv;
        h.Ap = fv + 3 * h.npair * pv;
        h.v = fv + 4 * h.npair * pv;
    }
    const int nsys = h.nsys;
    h.sc.nsys = nsys;
    h.sc.bn = c.take<double>(nsys);
    h.sc.rz = c.take<double>(2 * (size_t)nsys);
    h.sc.rr = c.take<double>(nsys);
    h.sc.pAp = c.take<double>(nsys);
    h.sc.alpha = c.take<double>(nsys);
    h.sc.beta = c.take<double>(nsys);
    h.sc.act = c.take<int>(nsys);
    h.sc.nconv = c.take<unsigned>(1);
    h.sc.itp = c.take<int>(1);
    const int nb = (int)((N + VB - 1) / VB);
    h.vpart = c.take<double>((size_t)2 * nsys * nb);
    h.vcnt = c.take<unsigned>(h.npair + 1);
    h.mpart = c.take<double>((size_t)nsys * pair_dot_blocks_max(h.L.nx, h.L.ny, h.L.nz));
    h.mcnt = c.take<unsigned>(nsys);
    h.err = c.take<int>(1);
    h.it_scr = c.take<int>(nsys);
    h.st_scr = c.take<int>(nsys);
    h.rel_scr = c.take<double>(nsys);
    h.nblk_pow = pow_blocks(N);
    const int npow = std::max(h.nset * h.nb0, h.nset);
    h.ppart = c.take<double>((size_t)2 * npow * std::max(h.nblk_pow, 64));
    h.rho0 = c.take<double>((size_t)h.nset * h.nb0);
    h.Pinv = c.take<double>((size_t)h.nset * GJ * GJ);
    int64_t nmax = 1;
    for (auto& b : h.box)
        for (int l = 0; l < b.nlev; ++l) nmax = std::max<int64_t>(nmax, b.lev[l].n);
    h.pw_x = c.take<float>((size_t)h.nset * nmax * 6);
    h.pw_y = c.take<float>((size_t)h.nset * nmax * 6);
    for (auto& b : h.box) {
        b.sys = c.take<int>(std::max(1, b.nsb));
        b.grp = c.take<int>((size_t)3 * std::max(1, b.ngrp));
        b.pent = c.take<int>((size_t)3 * std::max(1, b.npent));
        for (int l = 0; l < b.nlev; ++l) {
            auto& Lv = b.lev[l];
            const size_t vn = (size_t)std::max(1, b.nsb) * Lv.n * 6;
            Lv.A = c.take<float>((size_t)h.nset * STS * Lv.n);
            Lv.B = c.take<float>(vn);
            Lv.E = c.take<float>(vn);
            Lv.RB = c.take<float>(vn);
            if (l < b.nlev - 1) {
                Lv.Minv = c.take<float>((size_t)h.nset * 36 * Lv.n);
                Lv.Q = c.take<float>((size_t)Lv.n * 36);
                Lv.w = c.take<float>(h.nset);
                Lv.rho = c.take<double>(h.nset);
                Lv.X = c.take<float>(vn);
                Lv.X2 = c.take<float>(vn);
                Lv.T = c.take<float>(vn);
            }
        }
        b.Ainv = c.take<double>((size_t)h.nset * b.ncp * b.ncp);
        b.Ainv32 = c.take<float>((size_t)h.nset * b.ncp * b.ncp);
    }
}

// Geometry of one box (host): levels, grids, transfers below level 1 by modified Gram-Schmidt.
int box_geometry(lpm_amg::Box& b, int a, int coarse_max, int max_levels)
{
    for (int ax = 0; ax < 3; ++ax) {
        b.L[ax] = b.hi[ax] - b.lo[ax] + 1;
        b.nch[ax] = nchunks(b.L[ax], a);
    }
    auto& L1 = b.lev[0];
    for (int ax = 0; ax < 3; ++ax) L1.g[ax] = b.nch[ax];
    L1.n = b.nch[0] * b.nch[1] * b.nch[2];
    // closed-form R factors of the level-0 Gram-Schmidt (coarse rigid modes of every aggregate)
    std::vector<double> Bn((size_t)L1.n * 36, 0.0);
    for (int cz = 0; cz < b.nch[2]; ++cz)
        for (int cy = 0; cy < b.nch[1]; ++cy)
            for (int cx = 0; cx < b.nch[0]; ++cx) {
                const int c[3] = {cx, cy, cz};
                double C[3], s2[3], n = 1.0;
                for (int ax = 0; ax < 3; ++ax) {
                    int s0, w;
                    chunk_range(c[ax], a, b.nch[ax], b.L[ax], s0, w);
                    C[ax] = s0 + 0.5 * (w - 1) - 0.5 * (b.L[ax] - 1);
                    s2[ax] = (w * (double)w - 1.0) / 12.0;
                    n *= w;
                }
                const double sq = std::sqrt(n);
                const double n3 = std::sqrt(n * (s2[0] + s2[1])), n4 = std::sqrt(n * (s2[1] + s2[2])),
                             n5 = std::sqrt(n * (s2[0] + s2[2]));
                // rank test of gmg._tentative: every Gram-Schmidt column above 1e-8 of the largest column norm
                const double v3 = std::sqrt(n3 * n3 + n * (C[0] * C[0] + C[1] * C[1]));
                const double v4 = std::sqrt(n4 * n4 + n * (C[1] * C[1] + C[2] * C[2]));
                const double v5 = std::sqrt(n5 * n5 + n * (C[0] * C[0] + C[2] * C[2]));
                const double scale = std::max(std::max(sq, v3), std::max(v4, v5));
                if (!(n3 > 1e-8 * scale && n4 > 1e-8 * scale && n5 > 1e-8 * scale)) return LPM_ERR_UNSUPPORTED;
                double* R = Bn.data() + (size_t)((cz * b.nch[1] + cy) * b.nch[0] + cx) * 36;
                R[0 * 6 + 0] = R[1 * 6 + 1] = R[2 * 6 + 2] = sq;
                R[0 * 6 + 3] = -sq * C[1];
                R[1 * 6 + 3] = sq * C[0];
                R[1 * 6 + 4] = -sq * C[2];
                R[2 * 6 + 4] = sq * C[1];
                R[0 * 6 + 5] = sq * C[2];
                R[2 * 6 + 5] = -sq * C[0];
                R[3 * 6 + 3] = n3;
                R[4 * 6 + 4] = n4;
                R[5 * 6 + 5] = n5;
            }
    b.nlev = 1;
    while (6LL * b.lev[b.nlev - 1].n > coarse_max && b.nlev - 1 < max_levels) {
        if (b.nlev >= AMG_MAXL) return LPM_ERR_UNSUPPORTED;
        auto& F = b.lev[b.nlev - 1];
        auto& C = b.lev[b.nlev];
        for (int ax = 0; ax < 3; ++ax) C.g[ax] = nchunks(F.g[ax], a);
        C.n = C.g[0] * C.g[1] * C.g[2];
        F.Qh.assign((size_t)F.n * 36, 0.0);
        std::vector<double> Bc((size_t)C.n * 36, 0.0), blk, Q;
        for (int J = 0; J < C.n; ++J) {
            const int c[3] = {J % C.g[0], (J / C.g[0]) % C.g[1], J / (C.g[0] * C.g[1])};
            int s0[3], w[3];
            for (int ax = 0; ax < 3; ++ax) chunk_range(c[ax], a, C.g[ax], F.g[ax], s0[ax], w[ax]);
            std::vector<int> mem;
            for (int z = 0; z < w[2]; ++z)
                for (int y = 0; y < w[1]; ++y)
                    for (int x = 0; x < w[0]; ++x)
                        mem.push_back(((s0[2] + z) * F.g[1] + s0[1] + y) * F.g[0] + s0[0] + x);
            const int k = 6 * (int)mem.size();
            blk.assign((size_t)k * 6, 0.0);
            Q.assign((size_t)k * 6, 0.0);
            for (size_t m = 0; m < mem.size(); ++m)
                for (int r = 0; r < 6; ++r)
                    for (int cc = 0; cc < 6; ++cc) blk[(m * 6 + r) * 6 + cc] = Bn[(size_t)mem[m] * 36 + r * 6 + cc];
            if (!mgs6(blk, k, Q.data(), Bc.data() + (size_t)J * 36, 1e-8)) return LPM_ERR_UNSUPPORTED;
            for (size_t m = 0; m < mem.size(); ++m)
                for (int r = 0; r < 6; ++r)
                    for (int cc = 0; cc < 6; ++cc) F.Qh[(size_t)mem[m] * 36 + r * 6 + cc] = Q[(m * 6 + r) * 6 + cc];
        }
        Bn.swap(Bc);
        ++b.nlev;
    }
    b.nc = 6 * b.lev[b.nlev - 1].n;
    if (b.nc > 6144) return LPM_ERR_UNSUPPORTED;  // dense coarsest level limited to 6144 unknowns
    b.ncp = (b.nc + GJ - 1) / GJ * GJ;
    return LPM_OK;
}

inline dim3 grid2(int64_t n, int threads, int y) { return dim3((unsigned)((n + threads - 1) / threads), (unsigned)y); }

PairArgs pair_base(const lpm_amg& h)
{
    PairArgs a{};
    a.nx = h.L.nx;
    a.ny = h.L.ny;
    a.nz = h.L.nz;
    a.N = h.L.N;
    a.Kn = h.Kn;
    a.Tv = h.Tv;
    a.err = h.err;
    return a;
}

LvView view(const lpm_amg::Level& Lv)
{
    return LvView{Lv.g[0], Lv.g[1], Lv.g[2], Lv.n, Lv.A, Lv.Minv, Lv.w};
}

// ----------------------------------------------------------------------------------------- the cycle (host)
struct CycleCtx {
    const lpm_amg* h;
    const lpm_amg::Box* b;
    const int* act;
    cudaStream_t st;
};

cudaError_t vc(const CycleCtx& C, int l, const float* rhs, float* out, int acc);

// coarse(l): E[l] = approximate solve with B[l] (one cycle, or gamma cycles from level w_from on)
cudaError_t coarse(const CycleCtx& C, int l)
{
    const auto& b = *C.b;
    const auto& Lv = b.lev[l];
    cudaError_t e = vc(C, l, Lv.B, Lv.E, 0);
    if (e != cudaSuccess || l == b.nlev - 1) return e;
    const int extra = (l + 1 >= C.h->o.w_from) ? C.h->o.gamma - 1 : 0;
    for (int g = 0; g < extra && e == cudaSuccess; ++g) {
        k_lv_op<1><<<grid2(Lv.n, LB, b.ngrp), LB, 0, C.st>>>(view(Lv), b.grp, b.sys, C.act, Lv.E, Lv.B, Lv.RB,
                                                                   0);
        e = vc(C, l, Lv.RB, Lv.E, 1);
    }
    return e == cudaSuccess ? cudaGetLastError() : e;
}

// vc(l, rhs): one cycle on level l (0-based index into lev), result written (acc: added) to out
cudaError_t vc(const CycleCtx& C, int l, const float* rhs, float* out, int acc)
{
    const auto& h = *C.h;
    const auto& b = *C.b;
    const auto& Lv = b.lev[l];
    const dim3 g = grid2(Lv.n, LB, b.nsb), gg = grid2(Lv.n, LB, b.ngrp);
    if (l == b.nlev - 1) {
        k_dense_apply<<<grid2(b.nc, DR, b.ngrp), 256, 0, C.st>>>(b.nc, b.ncp, b.Ainv32, b.grp, b.sys, C.act, rhs,
                                                                     out, acc);
        return cudaGetLastError();
    }
    const LvView V = view(Lv);
    float *x = Lv.X, *x2 = Lv.X2;
    k_lv_bj<<<g, LB, 0, C.st>>>(V, b.sys, h.rps, C.act, rhs, x);
    for (int k = 0; k < h.o.nu_c - 1; ++k) {
        k_lv_op<2><<<gg, LB, 0, C.st>>>(V, b.grp, b.sys, C.act, x, rhs, x2, 0);
        std::swap(x, x2);
    }
    k_lv_op<1><<<gg, LB, 0, C.st>>>(V, b.grp, b.sys, C.act, x, rhs, Lv.T, 0);
    const auto& Cl = b.lev[l + 1];
    k_lv_restrict<<<dim3(Lv.tr.tiles, b.nsb), 256, Lv.tr.smem, C.st>>>(Lv.g[0], Lv.g[1], Lv.g[2], Lv.n, Cl.g[0],
                                                                         Cl.g[1], Cl.g[2], h.o.agg, Lv.tr.tw, Lv.tr.th,
                                                                         Lv.Q, b.sys, C.act, Lv.T, Cl.B);
    cudaError_t e = coarse(C, l + 1);
    if (e != cudaSuccess) return e;
    k_lv_prolong<<<g, LB, 0, C.st>>>(Lv.g[0], Lv.g[1], Lv.g[2], Cl.g[0], Cl.g[1], Cl.g[2], h.o.agg, Lv.Q, b.sys, h.rps,
                                     C.act, Cl.E, x);
    for (int k = 0; k < h.o.nu_c; ++k) {
        const bool last = k == h.o.nu_c - 1;
        k_lv_op<2><<<gg, LB, 0, C.st>>>(V, b.grp, b.sys, C.act, x, rhs, last ? out : x2, last ? acc : 0);
        if (!last) std::swap(x, x2);
    }
    return cudaGetLastError();
}

// Finest-level cycle: v holds w m M r on entry; z (in Ap) = the preconditioned residual on exit.  dot: also r.z and
// the PCG beta step.
cudaError_t fine_cycle(const lpm_amg& h, const FcgScalars& sc, bool dot, cudaStream_t st)
{
    PairArgs a = pair_base(h);
    a.nsys = h.nsys;
    a.rhs_per_set = h.rps;
    a.npp = h.npp;
    a.npair = h.npair;
    a.zchunk = h.zchunk;
    a.variant = h.variant;
    a.act = sc.act;
    a.rhs = h.r;
    a.Ms = h.Ms;
    a.fbox = h.fbox;
    a.fw = h.fw;
    a.u = h.v;
    a.out = h.Ap;
    cudaError_t e = launch_sc_pair_mode(a, PM_RESID, st);
    if (e != cudaSuccess) return e;
    // boxes in parallel: fork after the residual, join before the smoothing epilogue
    const bool fork = h.bst.size() > 1;
    if (fork) {
        if ((e = cudaEventRecord(h.bev[0], st)) != cudaSuccess) return e;
        for (auto sb : h.bst)
            if ((e = cudaStreamWaitEvent(sb, h.bev[0], 0)) != cudaSuccess) return e;
    }
    for (size_t bi = 0; bi < h.box.size(); ++bi) {
        const auto& b = h.box[bi];
        if (b.nsb == 0) continue;
        cudaStream_t sb = fork ? h.bst[bi] : st;
        BoxDev B{};
        for (int ax = 0; ax < 3; ++ax) {
            B.lo[ax] = b.lo[ax];
            B.L[ax] = b.L[ax];
            B.nch[ax] = b.nch[ax];
        }
        B.n1 = b.lev[0].n;
        B.B1 = b.lev[0].B;
        B.E1 = b.lev[0].E;
        const dim3 ga((unsigned)((B.n1 + TB - 1) / TB), (unsigned)b.npent);
        k_restrict_agg<<<ga, TB, 0, sb>>>(B, h.o.agg, h.L.nx, h.L.ny, h.L.N, b.pent, b.sys, sc.act, h.Ap);
        CycleCtx C{&h, &b, sc.act, sb};
        if ((e = coarse(C, 0)) != cudaSuccess) return e;
        // lanes of other boxes are never written, so the boxes' prolongations may run concurrently
        B.E1 = b.lev[0].E;
        k_prolong0<<<dim3(b.t0.tiles, b.npent), 256, 0, sb>>>(B, h.o.agg, b.t0.tw, b.t0.th, h.L.nx, h.L.ny, h.L.N,
                                                              b.pent, b.sys, sc.act, h.v);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (fork) {
            if ((e = cudaEventRecord(h.bev[1 + bi], sb)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(st, h.bev[1 + bi], 0)) != cudaSuccess) return e;
        }
    }
    a.part = dot ? h.mpart : nullptr;
    a.cnt = h.mcnt;
    a.scv = sc;
    a.has_sc = dot ? 1 : 0;
    return launch_sc_pair_mode(a, dot ? PM_SMOOTH_DOT : PM_SMOOTH, st);
}

// ------------------------------------------------------------------------------------------- numeric setup
// Widest aggregate of a box (the last chunk of an axis is the widest).  The direct level-1 product covers boxes whose
// aggregates are at most GD_WMAX sites wide (a = 3: widths 3..5); wider aggregates are probed.
int box_wmax(const lpm_amg::Box& b, int a)
{
    int wm = 1;
    for (int ax = 0; ax < 3; ++ax) {
        int s0, w;
        chunk_range(b.nch[ax] - 1, a, b.nch[ax], b.L[ax], s0, w);
        wm = std::max(wm, w);
    }
    return wm;
}

// Opt-in to k_galerkin0's dynamic shared memory (its largest size), once per device.
cudaError_t galerkin0_attr()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if ((done.load() >> dev) & 1ull) return cudaSuccess;
    e = cudaFuncSetAttribute(k_galerkin0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gd_smem(GD_WMAX));
    if (e == cudaSuccess) done.fetch_or(1ull << dev);
    return e;
}

int amg_setup(lpm_amg& h, const float* Kn, const float* Tv, const float* Minv, cudaStream_t st)
{
    const int64_t N = h.L.N;
    // The cycle's operator reads the handle's own copy of the coefficients: every buffer a captured iteration block
    // touches then stays at the same address from one setup to the next, so the graphs of the solve are reused
    // across setups (a new numeric setup only rewrites device memory those graphs read).
    h.ready = false;
    const size_t cb = sizeof(float) * (size_t)h.nset * 18 * N;
    cudaError_t e = cudaMemcpyAsync(h.Kn_own, Kn, cb, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.Tv_own, Tv, cb, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.err, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    h.Kn = h.Kn_own;
    h.Tv = h.Tv_own;
    k_repack_ms<<<grid2(N, VB, h.nset), VB, 0, st>>>(Minv, h.Ms, N);
    PairArgs base = pair_base(h);
    // ---- rho of the finest level: systems (set, k-th box), k < nb0
    {
        const int rpsp = h.nb0, nppp = (rpsp + 1) / 2, nsp = h.nset * rpsp;
        const PairGeom G{N, h.L.nx, h.L.ny, nsp, rpsp, nppp};
        float* x = h.xp;
        float* y = h.xp + (size_t)h.nset * nppp * N * 6;
        k_pow0_init<<<grid2(N, VB, h.nset * nppp), VB, 0, st>>>(G, h.pbox, h.Ms, x);
        PairArgs a = base;
        a.nsys = nsp;
        a.rhs_per_set = rpsp;
        a.npp = nppp;
        a.npair = h.nset * nppp;
        a.zchunk = pair_zchunk(h.L.nx, h.L.ny, h.L.nz, a.npair);
        a.variant = pair_variant(h.L.nx, h.L.ny, h.L.nz, a.npair);
        a.u = x;
        a.out = y;
        for (int it = 0; it < h.o.power_its; ++it) {
            if ((e = launch_sc_pair_mode(a, PM_NONE, st)) != cudaSuccess) return (int)e;
            k_pow0_step<<<dim3(h.nblk_pow, h.nset * nppp), VB, 0, st>>>(G, h.pbox, h.Ms, x, y, h.ppart);
        }
        k_pow_finish<<<(nsp + 7) / 8, 256, 0, st>>>(nsp, h.nblk_pow, h.ppart, h.rho0);
        k_fine_weights<<<(h.nsys + 127) / 128, 128, 0, st>>>(h.nsys, h.rps, h.nmask, h.nb0, h.box_of_mask, h.rho0,
                                                             h.o.omega, h.fw);
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    }
    for (auto& b : h.box) {
        auto& L1 = b.lev[0];
        BoxDev B{};
        for (int ax = 0; ax < 3; ++ax) {
            B.lo[ax] = b.lo[ax];
            B.L[ax] = b.L[ax];
            B.nch[ax] = b.nch[ax];
        }
        B.n1 = L1.n;
        if ((e = cudaMemsetAsync(L1.A, 0, sizeof(float) * (size_t)h.nset * STS * L1.n, st)) != cudaSuccess)
            return (int)e;
        const int wm = box_wmax(b, h.o.agg);
        if (wm <= GD_WMAX) {
            // ---- level 1 directly from the bonds
            if ((e = galerkin0_attr()) != cudaSuccess) return (int)e;
            k_galerkin0<<<dim3((unsigned)L1.n, h.nset), GD_T, gd_smem(wm), st>>>(B, h.o.agg, wm, h.L.nx, h.L.ny,
                                                                                h.L.nz, N, h.Kn, h.Tv, L1.A);
            if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        } else {
            // ---- level 1 by probing: 27 colour classes x 6 modes in chunks of PCOL colours
            float* pv = h.xp;
            float* py = h.xp + (size_t)h.nset * PNP * N * 6;
            PairArgs a = base;
            a.nsys = h.nset * PQ;
            a.rhs_per_set = PQ;
            a.npp = PNP;
            a.npair = h.nset * PNP;
            a.zchunk = h.zchunk_probe;
            a.variant = pair_variant(h.L.nx, h.L.ny, h.L.nz, a.npair);
            a.u = pv;
            a.out = py;
            if ((e = cudaMemsetAsync(pv, 0, sizeof(float) * (size_t)h.nset * PNP * N * 6, st)) != cudaSuccess)
                return (int)e;
            for (int chunk = 0; chunk < 27 / PCOL; ++chunk) {
                k_probe_gen<<<grid2(N, VB, h.nset * PNP), VB, 0, st>>>(B, h.o.agg, h.L.nx, h.L.ny, N, chunk, pv);
                if ((e = launch_sc_pair_mode(a, PM_NONE, st)) != cudaSuccess) return (int)e;
                k_restrict_probe<<<dim3(b.t0.tiles, h.nset * PNP), 256, b.t0.smem, st>>>(
                    B, h.o.agg, b.t0.tw, b.t0.th, h.L.nx, h.L.ny, N, py, chunk, L1.A);
            }
            if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        }
        // ---- levels below: block inverses, rho, Galerkin products
        for (int l = 0; l < b.nlev - 1; ++l) {
            auto& Lv = b.lev[l];
            auto& Cl = b.lev[l + 1];
            k_lv_diag_inv<<<grid2(Lv.n, 128, h.nset), 128, 0, st>>>(Lv.n, h.nset, Lv.A, Lv.Minv);
            k_pow_lv_init<<<grid2(Lv.n, 128, h.nset), 128, 0, st>>>(Lv.n, l + 1, Lv.Minv, h.pw_x);
            const int nbl = std::max(1, std::min(64, (Lv.n + LB - 1) / LB));
            for (int it = 0; it < h.o.power_its; ++it) {
                k_lv_op<0><<<grid2(Lv.n, LB, h.nset), LB, 0, st>>>(view(Lv), h.pgrp, nullptr, nullptr, h.pw_x,
                                                                   nullptr, h.pw_y, 0);
                k_pow_lv_step<<<dim3(nbl, h.nset), LB, 0, st>>>(Lv.n, Lv.Minv, h.pw_x, h.pw_y, h.ppart);
            }
            k_pow_finish<<<(h.nset + 7) / 8, 256, 0, st>>>(h.nset, nbl, h.ppart, Lv.rho);
            k_level_weights<<<(h.nset + 127) / 128, 128, 0, st>>>(h.nset, Lv.rho, h.o.omega, Lv.w);
            k_galerkin<<<dim3(Cl.n, h.nset), 256, 0, st>>>(Lv.g[0], Lv.g[1], Lv.g[2], Cl.g[0], Cl.g[1], Cl.g[2],
                                                           h.o.agg, Lv.A, Lv.Q, Cl.A);
            if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        }
        // ---- dense coarsest level: assemble, symmetrise, invert
        const auto& Lc = b.lev[b.nlev - 1];
        if ((e = cudaMemsetAsync(b.Ainv, 0, sizeof(double) * (size_t)h.nset * b.ncp * b.ncp, st)) != cudaSuccess)
            return (int)e;
        k_dense_build<<<dim3((unsigned)((std::max(Lc.n, b.ncp) + 127) / 128), 27, h.nset), 128, 0, st>>>(
            Lc.g[0], Lc.g[1], Lc.g[2], b.ncp, Lc.A, b.Ainv);
        k_dense_sym<<<dim3((b.nc + 15) / 16, (b.nc + 15) / 16, h.nset), dim3(16, 16), 0, st>>>(b.nc, b.ncp, b.Ainv);
        const int nbk = b.ncp / GJ, ntl = (b.ncp + GT - 1) / GT;
        for (int K = 0; K < nbk; ++K) {
            k_gj_diag<<<h.nset, dim3(GJ, GJ), 0, st>>>(K, b.ncp, b.Ainv, h.Pinv);
            k_gj_row<<<dim3(nbk, h.nset), 256, 0, st>>>(K, b.ncp, b.Ainv, h.Pinv);
            k_gj_trail<<<dim3(ntl, ntl, h.nset), 256, 0, st>>>(K, b.ncp, b.Ainv);
            k_gj_col<<<dim3(nbk, h.nset), 256, 0, st>>>(K, b.ncp, b.Ainv, h.Pinv);
        }
        const int64_t ne = (int64_t)h.nset * b.ncp * b.ncp;
        k_to_f32<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(b.Ainv, b.Ainv32, ne);
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    }
    int err = 0;
    e = cudaMemcpyAsync(&err, h.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    if (err) return LPM_ERR_TIMEOUT;
    ++h.gen;
    h.ready = true;
    return LPM_OK;
}

// Preconditioner application z = M_amg r for every system (r, z: (nsys, N, 3) FP32).
int amg_apply(lpm_amg& h, const float* r, float* z, cudaStream_t st)
{
    const int64_t N = h.L.N;
    FcgScalars sc = h.sc;
    sc.iters = h.it_scr;
    sc.relres = h.rel_scr;
    sc.status = h.st_scr;
    sc.tols = nullptr;
    sc.itp = nullptr;
    cudaError_t e = cudaMemsetAsync(h.vcnt, 0, sizeof(unsigned) * (h.npair + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.sc.nconv, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.Ap, 0, sizeof(float) * (size_t)h.npair * N * 6, st);
    if (e != cudaSuccess) return (int)e;
    const PairGeom G{N, h.L.nx, h.L.ny, h.nsys, h.rps, h.npp};
    const int gx = std::max(1, std::min((int)((N + VB - 1) / VB), (2 * 4 * 148 + h.npair - 1) / h.npair));
    k_amg_init<<<dim3(gx, h.npair), VB, 0, st>>>(G, r, h.fbox, h.fw, h.Ms, h.r, h.v, h.p, h.xp, sc, h.vpart, h.vcnt,
                                                 0.0, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    if ((e = fine_cycle(h, sc, false, st)) != cudaSuccess) return (int)e;
    if ((e = pair_unpack(h.Ap, z, N, h.nsys, h.rps, st)) != cudaSuccess) return (int)e;
    return LPM_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------------- the PCG
int amg_pcg(lpm_amg* hp, const float* b, float* x, const lpm_cg_opts& o, int* iters, double* relres, int* status,
            cudaStream_t st)
{
    if (!hp || !hp->ready) return LPM_ERR_ARG;
    lpm_amg& h = *hp;
    if (o.maxit < 0 || o.check < 1 || o.poll < 1) return LPM_ERR_ARG;
    const int64_t N = h.L.N;
    FcgScalars sc = h.sc;
    sc.iters = iters;
    sc.relres = relres;
    sc.status = status;
    sc.tols = o.tol_sys;
    cudaError_t e = pair_prepare();
    if (e == cudaSuccess) e = cudaMemsetAsync(h.vcnt, 0, sizeof(unsigned) * (h.npair + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.mcnt, 0, sizeof(unsigned) * h.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.sc.nconv, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.sc.itp, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(h.err, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    const PairGeom G{N, h.L.nx, h.L.ny, h.nsys, h.rps, h.npp};
    const int gx = std::max(1, std::min((int)((N + VB - 1) / VB), (2 * 4 * 148 + h.npair - 1) / h.npair));
    const dim3 pg = grid2(N, VB, h.npair);
    k_amg_init<<<dim3(gx, h.npair), VB, 0, st>>>(G, b, h.fbox, h.fw, h.Ms, h.r, h.v, h.p, h.xp, sc, h.vpart, h.vcnt,
                                                 o.tol, o.precheck);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    // z0 = M r0, p0 = z0, r0.z0 (iteration 0 of the beta step)
    if ((e = fine_cycle(h, sc, true, st)) != cudaSuccess) return (int)e;
    k_amg_pupdate<<<pg, VB, 0, st>>>(G, h.Ap, h.p, h.xp, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    unsigned nconv = 0;
    e = cudaMemcpyAsync(&nconv, h.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;

    KmvTimer timer(o.prof, st);
    PairArgs a = pair_base(h);
    a.nsys = h.nsys;
    a.rhs_per_set = h.rps;
    a.npp = h.npp;
    a.npair = h.npair;
    a.zchunk = h.zchunk;
    a.variant = h.variant;
    a.act = sc.act;
    a.part = h.mpart;
    a.cnt = h.mcnt;
    a.scv = sc;
    a.has_sc = 1;
    a.u = h.p;
    a.out = h.Ap;
    auto one_iter = [&](int it, cudaStream_t s) -> cudaError_t {
        timer.begin(nconv == 0);
        cudaError_t ee = launch_sc_pair_mode(a, PM_DOT, s);
        timer.end();
        if (ee != cudaSuccess) return ee;
        k_amg_update<<<dim3(gx, h.npair), VB, 0, s>>>(G, it, o.check, o.maxit, o.tol, h.fbox, h.fw, h.Ms, h.r, h.Ap,
                                                      h.v, sc, h.vpart, h.vcnt);
        if ((ee = cudaGetLastError()) != cudaSuccess) return ee;
        if ((ee = fine_cycle(h, sc, true, s)) != cudaSuccess) return ee;
        k_amg_pupdate<<<pg, VB, 0, s>>>(G, h.Ap, h.p, h.xp, sc);
        return cudaGetLastError();
    };
    GraphKey key;
    key.ptr = {hp, b, x, o.tol_sys, h.Kn, h.Tv, iters, relres, status, nullptr};
    key.val = {3, (long long)h.id, 0, o.poll, o.check, o.maxit, h.zchunk, h.variant, 0, 0, 0, 0, 0, 0, 0, 0};
    double tolv = o.tol;
    std::memcpy(&key.val[8], &tolv, sizeof(double));
    int it = 1, rc = LPM_OK;
    while (it <= o.maxit && nconv < (unsigned)h.nsys) {
        const int block = std::min(o.poll - (it - 1) % o.poll, o.maxit - it + 1);
        const bool use_graph = !o.prof && block == o.poll;  // every kernel was launched once by the init cycle
        if ((e = run_iteration_block(use_graph, key, it, block, st, one_iter)) != cudaSuccess) return (int)e;
        it += block;
        e = cudaMemcpyAsync(&nconv, h.sc.nconv, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return (int)e;
        timer.collect();
    }
    timer.collect();
    if ((e = pair_unpack(h.xp, x, N, h.nsys, h.rps, st)) != cudaSuccess) return (int)e;
    int err = 0;
    e = cudaMemcpyAsync(&err, h.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    if (err) rc = LPM_ERR_TIMEOUT;
    return rc;
}

bool amg_matches(const lpm_amg* h, const Lattice& L, const Batch& bt)
{
    return h && h->ready && L.dim == 3 && L.nbr == nullptr && L.nx == h->L.nx && L.ny == h->L.ny && L.nz == h->L.nz &&
           bt.nsys == h->nsys && bt.rhs_per_set == h->rps && bt.nmask == h->nmask;
}

}  // namespace lpm

// ================================================================================================ C ABI
using namespace lpm;

extern "C" {

void lpm_amg_default_opts(lpm_amg_opts* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->agg = 3;
    o->coarse_max = 1000;
    o->max_levels = 8;
    o->nu = 1;
    o->nu_c = 1;
    o->gamma = 2;
    o->w_from = 1;
    o->power_its = 5;
    o->omega = 1.32;
    o->rho0_per_box = 0;
}

int lpm_amg_create(const lpm_lattice* lat, const lpm_batch* batch, const int32_t* boxes, int32_t nbox,
                   const int32_t* box_of_mask, const lpm_amg_opts* opts, lpm_amg** out)
{
    if (!lat || !batch || !boxes || !box_of_mask || !opts || !out) return LPM_ERR_ARG;
    *out = nullptr;
    if (lat->dim != 3 || lat->nbr != nullptr || (int64_t)lat->nx * lat->ny * lat->nz != lat->n)
        return LPM_ERR_UNSUPPORTED;
    if (batch->nsys < 1 || batch->rhs_per_set < 1 || batch->nmask < 1) return LPM_ERR_ARG;
    if (nbox < 1 || nbox > AMG_MAXBOX) return LPM_ERR_UNSUPPORTED;
    const lpm_amg_opts& o = *opts;
    if (o.agg < 3 || o.agg > 6 || o.coarse_max < 6 || o.max_levels < 0 || o.max_levels > AMG_MAXL - 1 || o.nu != 1 ||
        o.nu_c < 1 || o.gamma < 1 || o.w_from < 1 || o.power_its < 1 || !(o.omega > 0.0))
        return LPM_ERR_UNSUPPORTED;
    auto h = new (std::nothrow) lpm_amg();
    if (!h) return LPM_ERR_ARG;
    h->L = Lattice{3, lat->nx, lat->ny, lat->nz, lat->n, nullptr};
    h->nsys = batch->nsys;
    h->rps = batch->rhs_per_set;
    h->nmask = batch->nmask;
    h->nset = (h->nsys + h->rps - 1) / h->rps;
    h->npp = (h->rps + 1) / 2;
    h->npair = h->nset * h->npp;
    h->nbox = nbox;
    h->o = o;
    h->nb0 = o.rho0_per_box ? nbox : 1;
    if (h->npair > 65535 || h->nset * PNP > 65535 || h->nset * PQ > 65535) {
        delete h;
        return LPM_ERR_UNSUPPORTED;
    }
    cudaGetDevice(&h->dev);
    h->id = g_amg_ids.fetch_add(1);
    h->box.resize(nbox);
    h->box_of_mask_h.assign(box_of_mask, box_of_mask + h->nmask);
    for (int m = 0; m < h->nmask; ++m)
        if (box_of_mask[m] < 0 || box_of_mask[m] >= nbox) {
            delete h;
            return LPM_ERR_ARG;
        }
    const int dims[3] = {lat->nx, lat->ny, lat->nz};
    for (int k = 0; k < nbox; ++k) {
        auto& b = h->box[k];
        for (int ax = 0; ax < 3; ++ax) {
            b.lo[ax] = boxes[6 * k + ax];
            b.hi[ax] = boxes[6 * k + 3 + ax];
            if (b.lo[ax] < 0 || b.hi[ax] >= dims[ax] || b.hi[ax] < b.lo[ax]) {
                delete h;
                return LPM_ERR_ARG;
            }
        }
        const int rc = box_geometry(b, o.agg, o.coarse_max, o.max_levels);
        if (rc != LPM_OK) {
            delete h;
            return rc;
        }
        b.t0 = tile_shape(b.nch, b.L, o.agg, 12);
        for (int l = 0; l + 1 < b.nlev; ++l) b.lev[l].tr = tile_shape(b.lev[l + 1].g, b.lev[l].g, o.agg, 6);
    }
    if (!pair_supported(lat->nx)) {  // the finest level runs on the pair-packed TMA operator
        delete h;
        return LPM_ERR_UNSUPPORTED;
    }
    std::vector<int> fbox((size_t)6 * h->nsys), sbox(h->nsys), sidx(h->nsys);
    for (int s = 0; s < h->nsys; ++s) {
        const int k = box_of_mask[s % h->nmask];
        sbox[s] = k;
        sidx[s] = (int)h->box[k].sys_h.size();
        h->box[k].sys_h.push_back(s);
        for (int ax = 0; ax < 3; ++ax) {
            fbox[6 * s + ax] = h->box[k].lo[ax];
            fbox[6 * s + 3 + ax] = h->box[k].hi[ax];
        }
    }
    for (int k = 0; k < nbox; ++k) {
        auto& b = h->box[k];
        b.nsb = (int)b.sys_h.size();
        for (int j = 0; j < b.nsb; ++j) {  // systems of one set are consecutive in the list
            const int set = b.sys_h[j] / h->rps;
            if (!b.grp_h.empty() && b.grp_h[b.grp_h.size() - 3] == set)
                ++b.grp_h.back();
            else
                b.grp_h.insert(b.grp_h.end(), {set, j, 1});
        }
        for (int pr = 0; pr < h->npair; ++pr) {
            const int set = pr / h->npp, jp = pr % h->npp;
            int jl[2] = {-1, -1};
            for (int l = 0; l < 2; ++l) {
                const int js = 2 * jp + l, s = set * h->rps + js;
                if (js < h->rps && s < h->nsys && sbox[s] == k) jl[l] = sidx[s];
            }
            if (jl[0] >= 0 || jl[1] >= 0) b.pent_h.insert(b.pent_h.end(), {pr, jl[0], jl[1]});
        }
        b.ngrp = (int)b.grp_h.size() / 3;
        b.npent = (int)b.pent_h.size() / 3;
        if (b.nsb > 65535 || b.npent > 65535) {
            delete h;
            return LPM_ERR_UNSUPPORTED;
        }
    }
    std::vector<int> pgrp;
    for (int s = 0; s < h->nset; ++s) pgrp.insert(pgrp.end(), {s, s, 1});
    std::vector<int> pbox((size_t)6 * h->nset * h->nb0);
    for (int s = 0; s < h->nset; ++s)
        for (int k = 0; k < h->nb0; ++k)
            for (int ax = 0; ax < 3; ++ax) {
                pbox[6 * (s * h->nb0 + k) + ax] = h->box[k].lo[ax];
                pbox[6 * (s * h->nb0 + k) + 3 + ax] = h->box[k].hi[ax];
            }
    Carver2 sizing{nullptr, 0};
    carve_amg(*h, sizing);
    h->bytes = sizing.off + 256;
    if (cudaMalloc(&h->mem, h->bytes) != cudaSuccess) {
        cudaGetLastError();
        h->mem = nullptr;
        delete h;
        return LPM_ERR_WORKSPACE;
    }
    Carver2 c{static_cast<char*>(h->mem), 0};
    carve_amg(*h, c);
    cudaError_t e = cudaMemcpy(h->box_of_mask, box_of_mask, sizeof(int) * h->nmask, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->fbox, fbox.data(), sizeof(int) * fbox.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->pbox, pbox.data(), sizeof(int) * pbox.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->pgrp, pgrp.data(), sizeof(int) * pgrp.size(), cudaMemcpyHostToDevice);
    for (int k = 0; k < nbox && e == cudaSuccess; ++k) {
        auto& b = h->box[k];
        if (b.nsb) e = cudaMemcpy(b.sys, b.sys_h.data(), sizeof(int) * b.nsb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && b.ngrp)
            e = cudaMemcpy(b.grp, b.grp_h.data(), sizeof(int) * b.grp_h.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && b.npent)
            e = cudaMemcpy(b.pent, b.pent_h.data(), sizeof(int) * b.pent_h.size(), cudaMemcpyHostToDevice);
        for (int l = 0; l < b.nlev - 1 && e == cudaSuccess; ++l) {
            std::vector<float> q(b.lev[l].Qh.begin(), b.lev[l].Qh.end());
            e = cudaMemcpy(b.lev[l].Q, q.data(), sizeof(float) * q.size(), cudaMemcpyHostToDevice);
        }
    }
    if (e != cudaSuccess) {
        delete h;
        return (int)e;
    }
    h->zchunk = pair_zchunk(h->L.nx, h->L.ny, h->L.nz, h->npair);
    h->variant = pair_variant(h->L.nx, h->L.ny, h->L.nz, h->npair);
    h->zchunk_probe = pair_zchunk(h->L.nx, h->L.ny, h->L.nz, h->nset * PNP);
    int nused = 0;
    for (auto& b : h->box) nused += b.nsb > 0;
    if (nused > 1) {
        h->bst.assign(nbox, nullptr);
        h->bev.assign(1 + nbox, nullptr);
        for (int k = 0; k < nbox && e == cudaSuccess; ++k)
            e = cudaStreamCreateWithFlags(&h->bst[k], cudaStreamNonBlocking);
        for (int k = 0; k < 1 + nbox && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&h->bev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            delete h;
            return (int)e;
        }
    }
    *out = h;
    return LPM_OK;
}

void lpm_amg_destroy(lpm_amg* h)
{
    if (!h) return;
    int cur = 0;
    const int dev = h->dev;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaDeviceSynchronize();
    delete h;
    if (cur != dev) cudaSetDevice(cur);
}

int lpm_amg_setup(lpm_amg* h, const float* Kn32, const float* Tv32, const float* Minv32, void* stream)
{
    if (!h || !Kn32 || !Tv32 || !Minv32) return LPM_ERR_ARG;
    if (!tma_aligned(Kn32, Tv32, Kn32)) return LPM_ERR_ARG;
    // pair tiles follow the autotuner if it has recorded this shape since create
    h->zchunk = pair_zchunk(h->L.nx, h->L.ny, h->L.nz, h->npair);
    h->variant = pair_variant(h->L.nx, h->L.ny, h->L.nz, h->npair);
    return amg_setup(*h, Kn32, Tv32, Minv32, static_cast<cudaStream_t>(stream));
}

int lpm_amg_set_rho0(lpm_amg* h, const double* rho0_host, void* stream)
{
    if (!h || !h->ready || !rho0_host) return LPM_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(h->rho0, rho0_host, sizeof(double) * h->nset * h->nb0, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return (int)e;
    k_fine_weights<<<(h->nsys + 127) / 128, 128, 0, st>>>(h->nsys, h->rps, h->nmask, h->nb0, h->box_of_mask, h->rho0,
                                                          h->o.omega, h->fw);
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? LPM_OK : (int)e;
}

int lpm_amg_get_rho0(const lpm_amg* h, double* rho0_host)
{
    if (!h || !h->ready || !rho0_host) return LPM_ERR_ARG;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(rho0_host, h->rho0, sizeof(double) * h->nset * h->nb0, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LPM_OK : (int)e;
}

int lpm_amg_apply(lpm_amg* h, const float* r, float* z, void* stream)
{
    if (!h || !h->ready || !r || !z) return LPM_ERR_ARG;
    return amg_apply(*h, r, z, static_cast<cudaStream_t>(stream));
}

int lpm_amg_pcg_f32(lpm_amg* h, const float* b, float* x, const lpm_cg_opts* opts, int32_t* iters, double* relres,
                    int32_t* status, void* stream)
{
    if (!h || !b || !x || !opts || !iters || !relres || !status) return LPM_ERR_ARG;
    return amg_pcg(h, b, x, *opts, iters, relres, status, static_cast<cudaStream_t>(stream));
}

int lpm_amg_info(const lpm_amg* h, int32_t box, int32_t* nlev, int32_t* grids, int64_t* device_bytes)
{
    if (!h || box < 0 || box >= h->nbox) return LPM_ERR_ARG;
    const auto& b = h->box[box];
    if (nlev) *nlev = b.nlev;
    if (grids)
        for (int l = 0; l < b.nlev; ++l)
            for (int ax = 0; ax < 3; ++ax) grids[3 * l + ax] = b.lev[l].g[ax];
    if (device_bytes) *device_bytes = (int64_t)h->bytes;
    return LPM_OK;
}

int lpm_amg_get_level(const lpm_amg* h, int32_t box, int32_t set, int32_t level, float* A_host, double* rho_host,
                      float* fw_host)
{
    if (!h || !h->ready || box < 0 || box >= h->nbox || set < 0 || set >= h->nset) return LPM_ERR_ARG;
    const auto& b = h->box[box];
    if (level < 1 || level > b.nlev) return LPM_ERR_ARG;
    const auto& Lv = b.lev[level - 1];
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess && A_host) {
        std::vector<float> t((size_t)STS * Lv.n);
        e = cudaMemcpy(t.data(), Lv.A + (size_t)set * STS * Lv.n, sizeof(float) * t.size(), cudaMemcpyDeviceToHost);
        // the full stencil (A_host: n x 27 x 6 x 6); directions whose neighbour lies off the grid stay zero
        std::fill(A_host, A_host + (size_t)Lv.n * ST, 0.f);
        for (int I = 0; I < Lv.n; ++I) {
            const int i0 = I % Lv.g[0], i1 = (I / Lv.g[0]) % Lv.g[1], i2 = I / (Lv.g[0] * Lv.g[1]);
            for (int d = 0; d < 27; ++d) {
                const int j0 = i0 + d % 3 - 1, j1 = i1 + (d / 3) % 3 - 1, j2 = i2 + d / 9 - 1;
                if (j0 < 0 || j0 >= Lv.g[0] || j1 < 0 || j1 >= Lv.g[1] || j2 < 0 || j2 >= Lv.g[2]) continue;
                const int J = (j2 * Lv.g[1] + j1) * Lv.g[0] + j0;
                for (int r = 0; r < 6; ++r)
                    for (int c = 0; c < 6; ++c)
                        A_host[(size_t)I * ST + d * 36 + r * 6 + c] =
                            d >= 13 ? t[(size_t)((d - 13) * 36 + r * 6 + c) * Lv.n + I]
                                    : t[(size_t)((13 - d) * 36 + c * 6 + r) * Lv.n + J];
            }
        }
    }
    if (e == cudaSuccess && rho_host) {
        if (level < b.nlev)
            e = cudaMemcpy(rho_host, Lv.rho + set, sizeof(double), cudaMemcpyDeviceToHost);
        else
            *rho_host = 0.0;
    }
    if (e == cudaSuccess && fw_host) e = cudaMemcpy(fw_host, h->fw, sizeof(float) * h->nsys, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LPM_OK : (int)e;
}

}  // extern "C"
