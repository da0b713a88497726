// Fused single-pass square-lattice operator on one tile of a full 2D box.
//
// The exact-Hessian g-form of timing/t2d/solver2d.py:269-305 needs, at particle i, the shell sums of i and of its
// eight neighbours, and those need the displacements of the neighbours' neighbours.  Here a 256-thread block stages
// the displacements of a 32 x 8 tile plus a 2-site halo in shared memory, forms the shell sums of the tile plus a
// 1-site ring there, and then the forces of the tile: one pass over global memory (displacements once, coefficients
// from L1/L2) instead of the two passes and the per-particle shell-sum round trip of the generic kernels.  The
// arithmetic is that of shell_sums_at / force_at (lpm_stencil.cuh), term for term.
#pragma once
#include "lpm_stencil.cuh"

namespace lpm {
namespace sqtile {

using stencil::Slots;

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int UW = TX + 4, UH = TY + 4;  // staged displacements: tile + 2-site halo
constexpr int SW = TX + 2, SH = TY + 2;  // shell sums: tile + 1-site ring

template <typename T>
struct Smem {
    T u[UH * UW * 2];
    T st[SH * SW * 4];
};

__host__ __device__ inline int tiles_x(int nx) { return (nx + TX - 1) / TX; }
__host__ __device__ inline int tiles_y(int ny) { return (ny + TY - 1) / TY; }

// Stage the displacements of the tile at (x0, y0) and its 2-site halo: load(q, v) fetches particle q's two
// components; sites outside the box are zero (never read as bonds).
template <typename T, class LD>
__device__ __forceinline__ void stage(int nx, int ny, int x0, int y0, const LD& load, Smem<T>& sm)
{
    for (int e = threadIdx.x; e < UH * UW; e += NT) {
        const int gx = x0 - 2 + e % UW, gy = y0 - 2 + e / UW;
        T v[2] = {T(0), T(0)};
        if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) load((int64_t)gy * nx + gx, v);
        sm.u[2 * e] = v[0];
        sm.u[2 * e + 1] = v[1];
    }
}

// Coefficient accessors address a site by its ring coordinates (lx, ly) = (x - x0 + 1, y - y0 + 1), 0 <= lx < SW,
// 0 <= ly < SH: the tile and its 1-site ring, where every coefficient a tile's forces and shell sums read lives.
template <typename T>
struct GlobalCoef {  // a coefficient set in global memory (any layout)
    const T* c;
    CoefLayout cl;
    int nx, x0, y0;
    __device__ __forceinline__ T operator()(int lx, int ly, int k) const
    {
        return c[((int64_t)(y0 - 1 + ly) * nx + (x0 - 1 + lx)) * cl.site_stride + k * cl.slot_stride];
    }
};
template <typename T>
struct SoaCoef {  // the packed layout in global memory: slot k of site q at c[k * N + q]
    const T* c;
    int64_t N;
    int64_t o0;  // site index of ring coordinates (0, 0), (y0 - 1) * nx + x0 - 1 (negative on the first row)
    int nx;
    __device__ __forceinline__ SoaCoef() = default;
    __device__ __forceinline__ SoaCoef(const T* c_, int64_t N_, int nx_, int x0, int y0)
        : c(c_), N(N_), o0((int64_t)(y0 - 1) * nx_ + (x0 - 1)), nx(nx_)
    {
    }
    // the site part in 32 bits (ly * nx + lx < 2^31 for any box the library accepts) and one 64-bit slot offset
    __device__ __forceinline__ T operator()(int lx, int ly, int k) const { return c[o0 + (ly * nx + lx) + k * N]; }
};
template <typename T>
struct SharedCoef {  // the ring region's coefficients staged in shared memory, slot-major
    const T* c;
    __device__ __forceinline__ T operator()(int lx, int ly, int k) const { return c[k * (SH * SW) + ly * SW + lx]; }
};

// Shell sums {S^0, S^1, TS^0, TS^1} of the tile and its 1-site ring from the staged displacements (zero outside the
// box).  tv(lx, ly, k): Tv of slot k of a ring site.
template <typename T, class TVA>
__device__ __forceinline__ void sums(int nx, int ny, int x0, int y0, const TVA& tv, Smem<T>& sm)
{
    using S = Slots<2>;
    for (int e = threadIdx.x; e < SH * SW; e += NT) {
        const int lx = e % SW, ly = e / SW;
        const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
        T s0 = 0, s1 = 0, t0 = 0, t1 = 0;
        if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
            const int c = (ly + 1) * UW + (lx + 1);
            const T ui[2] = {sm.u[2 * c], sm.u[2 * c + 1]};
#pragma unroll
            for (int k = 0; k < S::NN; ++k) {
                const int qx = gx + S::dx(k), qy = gy + S::dy(k);
                if (qx < 0 || qx >= nx || qy < 0 || qy >= ny) continue;
                const int cq = c + S::dy(k) * UW + S::dx(k);
                const T uq[2] = {sm.u[2 * cq], sm.u[2 * cq + 1]};
                const T d = stencil::dl_from<T, 2>(k, uq, ui);
                const T tvk = tv(lx, ly, k);
                if (S::shell(k) == 0) {
                    s0 += d;
                    t0 += tvk * d;
                } else {
                    s1 += d;
                    t1 += tvk * d;
                }
            }
        }
        T* o = sm.st + 4 * e;
        o[0] = s0;
        o[1] = s1;
        o[2] = t0;
        o[3] = t1;
    }
}

// Force on this thread's particle of the tile (if it is in the box): emit(i, f, ui) receives the particle index, the
// force and the particle's staged displacement.  kn(lx, ly, k), tv(lx, ly, k): coefficients of the ring sites.
template <typename T, class KNA, class TVA, class EMIT>
__device__ __forceinline__ void forces(int nx, int ny, int x0, int y0, const KNA& kn, const TVA& tv,
                                       const Smem<T>& sm, const EMIT& emit)
{
    using S = Slots<2>;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int gx = x0 + tx, gy = y0 + ty;
    if (gx >= nx || gy >= ny) return;
    const int64_t i = (int64_t)gy * nx + gx;
    const int c = (ty + 2) * UW + (tx + 2);
    const int cs = (ty + 1) * SW + (tx + 1);
    const T ui[2] = {sm.u[2 * c], sm.u[2 * c + 1]};
    const T Si[2] = {sm.st[4 * cs], sm.st[4 * cs + 1]}, TSi[2] = {sm.st[4 * cs + 2], sm.st[4 * cs + 3]};
    T f[2] = {T(0), T(0)};
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        const int qx = gx + S::dx(k), qy = gy + S::dy(k);
        if (qx < 0 || qx >= nx || qy < 0 || qy >= ny) continue;
        const int c_ = S::shell(k);
        const int cq = c + S::dy(k) * UW + S::dx(k);
        const int csq = cs + S::dy(k) * SW + S::dx(k);
        const T uq[2] = {sm.u[2 * cq], sm.u[2 * cq + 1]};
        const T d = stencil::dl_from<T, 2>(k, uq, ui);
        const T Sq[2] = {sm.st[4 * csq], sm.st[4 * csq + 1]}, TSq[2] = {sm.st[4 * csq + 2], sm.st[4 * csq + 3]};
        const T knk = kn(tx + 1, ty + 1, k), tvk = tv(tx + 1, ty + 1, k);
        const int qlx = tx + 1 + S::dx(k), qly = ty + 1 + S::dy(k);
        const T knq = kn(qlx, qly, k ^ 1), tvq = tv(qlx, qly, k ^ 1);
        const T F = (knk + knq) * d + T(0.5) * (tvk * Si[c_] + TSi[c_]) + T(0.5) * (tvq * Sq[c_] + TSq[c_]);
        const T Fw = F * bond_w<T>(c_);
        f[0] -= T(S::dx(k)) * Fw;
        f[1] -= T(S::dy(k)) * Fw;
    }
    emit(i, f, ui);
}

// Stage the coefficients of the tile and its 1-site ring (slot-major, zero outside the box) for SharedCoef.  The
// reads run along the contiguous direction of the layout: in the packed layout (unit site stride) a ring row of one
// slot is contiguous; in the reference layout (unit slot stride) a ring row's slots are, site after site, so
// consecutive threads take consecutive slots of a site.
template <typename T>
__device__ __forceinline__ void stage_coef(int nx, int ny, int x0, int y0, const T* __restrict__ c,
                                           const CoefLayout& cl, T* sc)
{
    if (cl.slot_stride == 1) {
#pragma unroll 4
        for (int e = threadIdx.x; e < 8 * SH * SW; e += NT) {
            const int ly = e / (8 * SW), rem = e - ly * (8 * SW);
            const int lx = rem >> 3, k = rem & 7;
            const int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
            sc[k * (SH * SW) + ly * SW + lx] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
                                                   ? c[((int64_t)gy * nx + gx) * cl.site_stride + k]
                                                   : T(0);
        }
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < 8 * SH * SW; e += NT) {
            const int k = e / (SH * SW), r = e - k * (SH * SW);
            const int gx = x0 - 1 + r % SW, gy = y0 - 1 + r / SW;
            sc[e] = (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
                        ? c[((int64_t)gy * nx + gx) * cl.site_stride + k * cl.slot_stride]
                        : T(0);
        }
    }
}

// Shared memory of a tile with both coefficient arrays staged (k_sq_fused): the displacement / shell-sum tile, then
// Kn and Tv of the tile and its ring, slot-major.
template <typename T>
struct CoefSmem {
    Smem<T> t;
    T kn[8 * SH * SW];
    T tv[8 * SH * SW];
};

}  // namespace sqtile
}  // namespace lpm
