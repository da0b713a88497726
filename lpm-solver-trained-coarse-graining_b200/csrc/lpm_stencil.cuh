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

template <typename T, int DIM>
__device__ __forceinline__ T dl_of(const T* __restrict__ us, int64_t i, int64_t q, int k, const T* ui)
{
    using S = Slots<DIM>;
    T d = T(S::dx(k)) * (us[DIM * q] - ui[0]) + T(S::dy(k)) * (us[DIM * q + 1] - ui[1]);
    if constexpr (DIM == 3) d += T(S::dz(k)) * (us[DIM * q + 2] - ui[2]);
    return d * bond_w<T>(S::shell(k));
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
