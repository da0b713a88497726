// Stencil helpers shared by the LPM kernels: slot traits, thread placement, implicit / tabulated neighbours.
#pragma once
#include "lpm_common.cuh"

namespace lpm {
namespace stencil {

constexpr int BX = 32, BY = 8;    // structured block
constexpr int TB = 256;           // table block

template <int DIM>
struct Slots;
template <>
struct Slots<3> {
    static constexpr int NN = 18;
    static __device__ __forceinline__ constexpr int dx(int k) { return sc_dx(k); }
    static __device__ __forceinline__ constexpr int dy(int k) { return sc_dy(k); }
    static __device__ __forceinline__ constexpr int dz(int k) { return sc_dz(k); }
    static __device__ __forceinline__ constexpr int shell(int k) { return sc_shell(k); }
};
template <>
struct Slots<2> {
    static constexpr int NN = 8;
    static __device__ __forceinline__ constexpr int dx(int k) { return sq_dx(k); }
    static __device__ __forceinline__ constexpr int dy(int k) { return sq_dy(k); }
    static __device__ __forceinline__ constexpr int dz(int) { return 0; }
    static __device__ __forceinline__ constexpr int shell(int k) { return sq_shell(k); }
};

// Where a thread sits: particle index, grid coordinates and system.
struct Site {
    int64_t i;
    int x, y, z;
    int s;
    bool ok;
};

template <int DIM>
struct GridNb {
    static constexpr bool structured = true;
    static constexpr int dim = DIM;
    int nx, ny, nz;
    __device__ __forceinline__ bool get(const Site& p, int k, int64_t& q) const
    {
        using S = Slots<DIM>;
        const int qx = p.x + S::dx(k), qy = p.y + S::dy(k), qz = p.z + S::dz(k);
        bool ok = qx >= 0 && qx < nx && qy >= 0 && qy < ny;
        if (DIM == 3) ok = ok && qz >= 0 && qz < nz;
        q = p.i + ((int64_t)S::dz(k) * ny + S::dy(k)) * nx + S::dx(k);
        return ok;
    }
};

template <int DIM>
struct TableNb {
    static constexpr bool structured = false;
    static constexpr int dim = DIM;
    const int32_t* nbr;
    __device__ __forceinline__ bool get(const Site& p, int k, int64_t& q) const
    {
        const int v = __ldg(nbr + p.i * Slots<DIM>::NN + k);
        q = v;
        return v >= 0;
    }
};

template <class NB>
__device__ __forceinline__ Site locate(int nx, int ny, int nz, int64_t N, int sys0)
{
    Site p;
    if constexpr (NB::structured) {
        p.x = blockIdx.x * BX + threadIdx.x;
        p.y = blockIdx.y * BY + threadIdx.y;
        p.z = blockIdx.z % nz;
        p.s = sys0 + blockIdx.z / nz;
        p.ok = p.x < nx && p.y < ny;
        p.i = ((int64_t)p.z * ny + p.y) * nx + p.x;
    } else {
        p.i = (int64_t)blockIdx.x * TB + threadIdx.x;
        p.x = p.y = p.z = 0;
        p.s = sys0 + blockIdx.y;
        p.ok = p.i < N;
    }
    return p;
}

template <class NB>
__device__ __forceinline__ int block_in_system(int nz)
{
    if constexpr (NB::structured)
        return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (blockIdx.z % nz));
    else
        return blockIdx.x;
}

// dL of slot k from the displacements of the particle (ui) and of its slot-k neighbour (uq): o_k.(u_q - u_i) / |o_k|.
template <typename T, int DIM>
__device__ __forceinline__ T dl_from(int k, const T* uq, const T* ui)
{
    using S = Slots<DIM>;
    T d = T(S::dx(k)) * (uq[0] - ui[0]) + T(S::dy(k)) * (uq[1] - ui[1]);
    if constexpr (DIM == 3) d += T(S::dz(k)) * (uq[2] - ui[2]);
    return d * bond_w<T>(S::shell(k));
}

template <typename T, int DIM>
__device__ __forceinline__ T dl_of(const T* __restrict__ us, int64_t i, int64_t q, int k, const T* ui)
{
    T uq[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) uq[a] = us[DIM * q + a];
    return dl_from<T, DIM>(k, uq, ui);
}

// Pass 1 of the operator at one particle (coarse3d/lin3d.py:98-124): o = {S^0, S^1, TS^0, TS^1} with
// S^c = sum_{k in c} dL_k and TS^c = sum_{k in c} Tv_k dL_k over the bonds that exist.  load(q, uq) fetches the DIM
// displacement components of particle q; tv points at slot 0 of the particle's Tv (slot k at tv[k * slot_stride]).
template <typename T, int DIM, class NB, class LD>
__device__ __forceinline__ void shell_sums_at(const NB& nb, const Site& p, const T* ui, const LD& load,
                                              const T* __restrict__ tv, int64_t slot_stride, T (&o)[4])
{
    using S = Slots<DIM>;
    T s0 = 0, s1 = 0, t0 = 0, t1 = 0;
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        T uq[DIM];
        load(q, uq);
        const T d = dl_from<T, DIM>(k, uq, ui);
        const T tvk = tv[k * slot_stride];
        if (S::shell(k) == 0) {
            s0 += d;
            t0 += tvk * d;
        } else {
            s1 += d;
            t1 += tvk * d;
        }
    }
    o[0] = s0;
    o[1] = s1;
    o[2] = t0;
    o[3] = t1;
}

// Pass 2 at one particle: f = sum_k F_k n_k from the shell sums of the particle (Si, TSi) and of its neighbours
// (sums(q, S, TS)).  SC, code-force form (coarse3d/lin3d.py:126-149):
//   F_k = 2 Kn_k dL_k + (TS_i^c + TS_q^c)/2 + Tv_k (S_i^c + S_q^c)/2.
// SQ, exact-Hessian g-form (timing/t2d/solver2d.py:269-305), which also needs the neighbour's own slot k^1:
//   F_k = (Kn_k + Kn_q,k^1) dL_k + (Tv_k S_i^c + TS_i^c)/2 + (Tv_q,k^1 S_q^c + TS_q^c)/2.
// kn / tv point at slot 0 of the particle's coefficients; kset / tset at the coefficient set (SQ only).
template <typename T, int DIM, class NB, class LD, class SUMS>
__device__ __forceinline__ void force_at(const NB& nb, const Site& p, const T* ui, const LD& load, const SUMS& sums,
                                         const T (&Si)[2], const T (&TSi)[2], const T* __restrict__ kn,
                                         const T* __restrict__ tv, const T* __restrict__ kset,
                                         const T* __restrict__ tset, const CoefLayout& cl, T (&f)[3])
{
    using S = Slots<DIM>;
    f[0] = f[1] = f[2] = T(0);
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        const int c = S::shell(k);
        T uq[DIM];
        load(q, uq);
        const T d = dl_from<T, DIM>(k, uq, ui);
        T Sq[2], TSq[2];
        sums(q, Sq, TSq);
        const T knk = kn[k * cl.slot_stride], tvk = tv[k * cl.slot_stride];
        T F;
        if constexpr (DIM == 3) {
            F = T(2) * knk * d + T(0.5) * (TSi[c] + TSq[c]) + T(0.5) * tvk * (Si[c] + Sq[c]);
        } else {
            const int64_t qo = (int64_t)q * cl.site_stride + (k ^ 1) * cl.slot_stride;
            const T knq = kset[qo], tvq = tset[qo];
            F = (knk + knq) * d + T(0.5) * (tvk * Si[c] + TSi[c]) + T(0.5) * (tvq * Sq[c] + TSq[c]);
        }
        // f += F n_k with n_k = -o_k w_k
        const T Fw = F * bond_w<T>(c);
        f[0] -= T(S::dx(k)) * Fw;
        f[1] -= T(S::dy(k)) * Fw;
        if constexpr (DIM == 3) f[2] -= T(S::dz(k)) * Fw;
    }
}

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
    using type = float4;
};
template <>
struct Vec4<double> {
    using type = double4;
};

template <typename T>
__device__ __forceinline__ void load4(const T* p, T& a, T& b, T& c, T& d)
{
    const typename Vec4<T>::type v = *reinterpret_cast<const typename Vec4<T>::type*>(p);
    a = v.x;
    b = v.y;
    c = v.z;
    d = v.w;
}


}  // namespace stencil
}  // namespace lpm
