// Shared device definitions of the LPM CUDA library: lattice slot tables, batch/coefficient addressing, reductions.
//
// Lattices (same slot order as the reference: coarse3d/geom3d.py:16-19, coarse2d/lin2d.py:21-22):
//   SC (3D, 18 slots): shell 0 = axial slots 0..5, shell 1 = face diagonals 6..17; slots pair as (k, k^1).
//   SQ (2D,  8 slots): shell 0 = axial slots 0..3, shell 1 = diagonals 4..7.
// Bond direction n_k = -o_k/|o_k| (o_k = neighbour offset), so dL_ik = n_k.(u_i - u_q) = (o_k.(u_q - u_i))/|o_k|.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lpm {

// ---------------------------------------------------------------------------------------------------- slot tables
__host__ __device__ constexpr int sc_dx(int k)
{
    constexpr int t[18] = {1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[k];
}
__host__ __device__ constexpr int sc_dy(int k)
{
    constexpr int t[18] = {0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[k];
}
__host__ __device__ constexpr int sc_dz(int k)
{
    constexpr int t[18] = {0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[k];
}
__host__ __device__ constexpr int sc_shell(int k) { return k < 6 ? 0 : 1; }

__host__ __device__ constexpr int sq_dx(int k)
{
    constexpr int t[8] = {1, -1, 0, 0, 1, -1, 1, -1};
    return t[k];
}
__host__ __device__ constexpr int sq_dy(int k)
{
    constexpr int t[8] = {0, 0, 1, -1, 1, -1, -1, 1};
    return t[k];
}
__host__ __device__ constexpr int sq_shell(int k) { return k < 4 ? 0 : 1; }

// 1/|o_k| for diagonal slots, as the reference computes it: 1/sqrt(2) in double (-offs / np.linalg.norm(offs)).
constexpr double INV_SQRT2 = 1.0 / 1.4142135623730951;

template <typename T>
__device__ __forceinline__ T bond_w(int shell)
{
    return shell == 0 ? T(1) : T(INV_SQRT2);
}

// ------------------------------------------------------------------------------------------ coefficient addressing
// Coefficient set c, particle i, slot k lives at base + c*set_stride + k*slot_stride + i*site_stride.
//   reference layout (N, NN):   slot_stride = 1,  site_stride = NN
//   packed SoA layout (NN, N):  slot_stride = N,  site_stride = 1
struct CoefLayout {
    int64_t set_stride;
    int64_t slot_stride;
    int64_t site_stride;
};

// -------------------------------------------------------------------------------------------------- batch layout
// A batch holds nsys systems (right-hand sides).  System s uses coefficient set s / rhs_per_set and DOF mask
// s % nmask (masks are uint8 per DOF, 1 = free).  Vectors are (nsys, N, d) contiguous.
struct Batch {
    int nsys;
    int rhs_per_set;
    int nmask;
};

// ------------------------------------------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of v over the block (any blockDim multiple of 32, <= 1024); result valid in thread 0.  Fixed order ->
// deterministic.  `sh` needs 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x * blockDim.y) >> 5;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    v = warp_sum(v);
    __syncthreads();
    if ((tid & 31) == 0) sh[tid >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (tid < 32) {
        r = tid < nw ? sh[tid] : 0.0;
        r = warp_sum(r);
    }
    (void)lane;
    (void)wid;
    return r;
}

template <typename T>
__device__ __forceinline__ bool finite_val(T v)
{
    return isfinite(v);
}

}  // namespace lpm
