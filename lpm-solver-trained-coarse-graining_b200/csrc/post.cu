// Post-processing and per-bond gradient kernels (FP64), plus coefficient packing and neighbour-table construction.
//
// Stress (computeStress with the opp-flag surface rule; coarse3d/lin3d.py:170-210, timing/t2d/solver2d.py:220-256):
//   sigma_i = sum_k (of_ik / V) l0_k F_ik n_k n_k^T,  of = 1/2 if all slots are bonds or slot k^1 is a bond, else 1,
//   F_ik the code-force bond force (both lattices).
// Energy (coarse3d/lin3d.py:213-236, coarse2d/lin2d.py:156-163): U_i = 1/2 sum_k Kn dL^2 + 1/2 sum_c S_c TS_c.
// Gradients of lam . K u w.r.t. the per-slot parameters (closed forms of the reference's autograd passes):
//   SC (code-force, coarse3d/torch_lpm3d.py:165-175):
//       d/dKn_ik = 2 dL(u)_ik (n_k.lam_i),  d/dTv_ik = 1/2 dL(u)_ik S_i^c(lam) + 1/2 (S_i^c(u) + S_q^c(u)) (n_k.lam_i)
//   SQ (exact Hessian, coarse2d/torch_lpm.py:173-191 + 34-51):
//       d/dKn_ik = dL(lam)_ik dL(u)_ik,     d/dTv_ik = 1/2 [dL(lam)_ik S_i^c(u) + dL(u)_ik S_i^c(lam)]
#include "lpm_kernels.h"
#include "lpm_stencil.cuh"

namespace lpm {

namespace {

using namespace stencil;

template <int DIM, class NB>
__device__ __forceinline__ bool full_site(const NB& nb, const Site& p)
{
    bool full = true;
#pragma unroll
    for (int k = 0; k < Slots<DIM>::NN; ++k) {
        int64_t q;
        full = full && nb.get(p, k, q);
    }
    return full;
}

template <int DIM, class NB>
__global__ void __launch_bounds__(256) k_stress(NB nb, int nx, int ny, int nz, int64_t N, int sys0,
                                                const double* __restrict__ u, const double* __restrict__ Kn,
                                                const double* __restrict__ Tv, CoefLayout cl, Batch bt,
                                                const double* __restrict__ st, const double* __restrict__ l0,
                                                double V, double* __restrict__ sig)
{
    using S = Slots<DIM>;
    constexpr int NC = DIM == 3 ? 6 : 3;
    const Site p = locate<NB>(nx, ny, nz, N, sys0);
    if (!p.ok) return;
    const double* us = u + (int64_t)p.s * N * DIM;
    const int64_t cbase = (int64_t)(p.s / bt.rhs_per_set) * cl.set_stride;
    const double* sts = st + (int64_t)p.s * N * 4;
    double ui[3];
#pragma unroll
    for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
    double Si[2], TSi[2];
    load4(sts + 4 * p.i, Si[0], Si[1], TSi[0], TSi[1]);
    const bool full = full_site<DIM>(nb, p);
    double out[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c] = 0.0;
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        int64_t qo;
        const double of = (full || nb.get(p, k ^ 1, qo)) ? 0.5 : 1.0;
        const int c = S::shell(k);
        const double d = dl_of<double, DIM>(us, p.i, q, k, ui);
        double Sq[2], TSq[2];
        load4(sts + 4 * q, Sq[0], Sq[1], TSq[0], TSq[1]);
        const int64_t io = cbase + p.i * cl.site_stride + k * cl.slot_stride;
        const double F = 2.0 * Kn[io] * d + 0.5 * (TSi[c] + TSq[c]) + 0.5 * Tv[io] * (Si[c] + Sq[c]);
        const double a = of / V * l0[k] * F;
        const double w = c == 0 ? 1.0 : INV_SQRT2;
        const double n0 = -S::dx(k) * w, n1 = -S::dy(k) * w, n2 = -S::dz(k) * w;
        if constexpr (DIM == 3) {
            out[0] += a * n0 * n0;
            out[1] += a * n1 * n1;
            out[2] += a * n2 * n2;
            out[3] += a * n1 * n2;
            out[4] += a * n0 * n2;
            out[5] += a * n0 * n1;
        } else {
            out[0] += a * n0 * n0;
            out[1] += a * n1 * n1;
            out[2] += a * n0 * n1;
        }
    }
    double* o = sig + ((int64_t)p.s * N + p.i) * NC;
#pragma unroll
    for (int c = 0; c < NC; ++c) o[c] = out[c];
}

template <int DIM, class NB>
__global__ void __launch_bounds__(256) k_energy(NB nb, int nx, int ny, int nz, int64_t N, int sys0,
                                                const double* __restrict__ u, const double* __restrict__ Kn,
                                                const double* __restrict__ Tv, CoefLayout cl, Batch bt,
                                                double* __restrict__ w)
{
    using S = Slots<DIM>;
    const Site p = locate<NB>(nx, ny, nz, N, sys0);
    if (!p.ok) return;
    const double* us = u + (int64_t)p.s * N * DIM;
    const int64_t cbase = (int64_t)(p.s / bt.rhs_per_set) * cl.set_stride;
    double ui[3];
#pragma unroll
    for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
    double e = 0.0, s[2] = {0.0, 0.0}, t[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        const double d = dl_of<double, DIM>(us, p.i, q, k, ui);
        const int64_t io = cbase + p.i * cl.site_stride + k * cl.slot_stride;
        e += 0.5 * Kn[io] * d * d;
        s[S::shell(k)] += d;
        t[S::shell(k)] += Tv[io] * d;
    }
    w[(int64_t)p.s * N + p.i] = e + 0.5 * (s[0] * t[0] + s[1] * t[1]);
}

// One thread per (coefficient set, particle); loops over the systems of the set.  st_u / st_l: shell sums of u and
// lam (nsys, N, 4) (SC only).
template <int DIM, class NB, bool HESS>
__global__ void __launch_bounds__(256) k_grad(NB nb, int nx, int ny, int nz, int64_t N, int nset,
                                              const double* __restrict__ u, const double* __restrict__ lam,
                                              Batch bt, const double* __restrict__ st_u,
                                              const double* __restrict__ st_l, double* __restrict__ gKn,
                                              double* __restrict__ gTv, int accumulate, int set0)
{
    using S = Slots<DIM>;
    constexpr int NN = S::NN;
    const Site p = locate<NB>(nx, ny, nz, N, set0);  // p.s = coefficient set
    if (!p.ok || p.s >= nset) return;
    double gk[NN], gt[NN];
#pragma unroll
    for (int k = 0; k < NN; ++k) gk[k] = gt[k] = 0.0;
    const int s_lo = p.s * bt.rhs_per_set;
    const int s_hi = min(bt.nsys, s_lo + bt.rhs_per_set);
    for (int s = s_lo; s < s_hi; ++s) {
        const double* us = u + (int64_t)s * N * DIM;
        const double* ls = lam + (int64_t)s * N * DIM;
        double ui[3], li[3];
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            ui[a] = us[DIM * p.i + a];
            li[a] = ls[DIM * p.i + a];
        }
        if constexpr (HESS) {
            double du[NN], dl[NN], su[2] = {0, 0}, sl[2] = {0, 0};
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                int64_t q;
                du[k] = dl[k] = 0.0;
                if (!nb.get(p, k, q)) continue;
                du[k] = dl_of<double, DIM>(us, p.i, q, k, ui);
                dl[k] = dl_of<double, DIM>(ls, p.i, q, k, li);
                su[S::shell(k)] += du[k];
                sl[S::shell(k)] += dl[k];
            }
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                const int c = S::shell(k);
                gk[k] += dl[k] * du[k];
                gt[k] += 0.5 * (dl[k] * su[c] + du[k] * sl[c]);
            }
        } else {
            double Sui[2], TSu[2], Sli[2], TSl[2];
            load4(st_u + ((int64_t)s * N + p.i) * 4, Sui[0], Sui[1], TSu[0], TSu[1]);
            load4(st_l + ((int64_t)s * N + p.i) * 4, Sli[0], Sli[1], TSl[0], TSl[1]);
#pragma unroll
            for (int k = 0; k < NN; ++k) {
                int64_t q;
                if (!nb.get(p, k, q)) continue;
                const int c = S::shell(k);
                const double d = dl_of<double, DIM>(us, p.i, q, k, ui);
                const double w = c == 0 ? 1.0 : INV_SQRT2;
                double nl = -S::dx(k) * li[0] - S::dy(k) * li[1];
                if constexpr (DIM == 3) nl -= S::dz(k) * li[2];
                nl *= w;
                double Suq[2], TSuq[2];
                load4(st_u + ((int64_t)s * N + q) * 4, Suq[0], Suq[1], TSuq[0], TSuq[1]);
                gk[k] += 2.0 * d * nl;
                gt[k] += 0.5 * d * Sli[c] + 0.5 * (Sui[c] + Suq[c]) * nl;
            }
        }
    }
    double* ok = gKn + ((int64_t)p.s * N + p.i) * NN;
    double* ot = gTv + ((int64_t)p.s * N + p.i) * NN;
#pragma unroll
    for (int k = 0; k < NN; ++k) {
        ok[k] = accumulate ? ok[k] + gk[k] : gk[k];
        ot[k] = accumulate ? ot[k] + gt[k] : gt[k];
    }
}

template <typename T>
__global__ void k_pack(const double* __restrict__ src, T* __restrict__ dst, int64_t N, int NN)
{
    const int c = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double* s = src + ((int64_t)c * N + i) * NN;
    T* d = dst + (int64_t)c * N * NN + i;
    for (int k = 0; k < NN; ++k) d[(int64_t)k * N] = (T)s[k];
}

template <int DIM>
__global__ void k_build_nbr(int nx, int ny, int nz, int64_t n, const int64_t* __restrict__ site_of,
                            const int64_t* __restrict__ sites, int64_t* __restrict__ nbr)
{
    using S = Slots<DIM>;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t site = sites[j];
    const int x = (int)(site % nx);
    const int y = (int)((site / nx) % ny);
    const int z = (int)(site / ((int64_t)nx * ny));
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        const int qx = x + S::dx(k), qy = y + S::dy(k), qz = z + S::dz(k);
        int64_t q = -1;
        if (qx >= 0 && qx < nx && qy >= 0 && qy < ny && qz >= 0 && qz < nz)
            q = site_of[((int64_t)qz * ny + qy) * nx + qx];
        nbr[j * S::NN + k] = q >= 0 ? q : -1;
    }
}

// Bond table of one specimen with voids on the full box: slot k of site i exists iff the geometric neighbour q is
// inside the box and both i and q are solid (cement3d/torch_v1.py:37-45, valid = gvalid & solid_i & solid_q).
template <int DIM>
__global__ void k_solid_nbr(int nx, int ny, int nz, const uint8_t* __restrict__ solid, int32_t* __restrict__ nbr)
{
    using S = Slots<DIM>;
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t b = blockIdx.y;
    const uint8_t* sb = solid + b * n;
    int32_t* o = nbr + (b * n + i) * S::NN;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((int64_t)nx * ny));
    const bool si = sb[i] != 0;
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        const int qx = x + S::dx(k), qy = y + S::dy(k), qz = z + S::dz(k);
        int32_t q = -1;
        if (si && qx >= 0 && qx < nx && qy >= 0 && qy < ny && qz >= 0 && qz < nz) {
            const int64_t qi = ((int64_t)qz * ny + qy) * nx + qx;
            if (sb[qi]) q = (int32_t)qi;
        }
        o[k] = q;
    }
}

template <int DIM, class NB, typename F>
cudaError_t per_system(NB, const Lattice& L, int nsys, cudaStream_t st, F&& launch)
{
    const int nz = DIM == 3 ? L.nz : 1;
    if constexpr (NB::structured) {
        const int chunk = 65535 / nz;
        for (int s0 = 0; s0 < nsys; s0 += chunk) {
            const int ns = nsys - s0 < chunk ? nsys - s0 : chunk;
            launch(dim3((L.nx + BX - 1) / BX, (L.ny + BY - 1) / BY, nz * ns), dim3(BX, BY), s0);
        }
    } else {
        for (int s0 = 0; s0 < nsys; s0 += 65535) {
            const int ns = nsys - s0 < 65535 ? nsys - s0 : 65535;
            launch(dim3((unsigned)((L.N + TB - 1) / TB), ns), dim3(TB), s0);
        }
    }
    (void)st;
    return cudaGetLastError();
}

template <int DIM, class NB>
cudaError_t run_stress(NB nb, const Lattice& L, const double* u, const double* Kn, const double* Tv,
                       const CoefLayout& cl, const Batch& bt, const double* l0, double V, double* sig, double* scratch,
                       cudaStream_t st)
{
    cudaError_t e = launch_kmv_sums(L, u, Tv, cl, bt, scratch, st);
    if (e != cudaSuccess) return e;
    const int nz = DIM == 3 ? L.nz : 1;
    return per_system<DIM>(nb, L, bt.nsys, st, [&](dim3 g, dim3 b, int s0) {
        k_stress<DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Kn, Tv, cl, bt, scratch, l0, V, sig);
    });
}

template <int DIM, class NB>
cudaError_t run_energy(NB nb, const Lattice& L, const double* u, const double* Kn, const double* Tv,
                       const CoefLayout& cl, const Batch& bt, double* w, cudaStream_t st)
{
    const int nz = DIM == 3 ? L.nz : 1;
    return per_system<DIM>(nb, L, bt.nsys, st, [&](dim3 g, dim3 b, int s0) {
        k_energy<DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Kn, Tv, cl, bt, w);
    });
}

template <int DIM, class NB>
cudaError_t run_grad(NB nb, const Lattice& L, const double* u, const double* lam, const double* Kn, const double* Tv,
                     const CoefLayout& cl, const Batch& bt, double* gKn, double* gTv, double* scratch, int acc,
                     cudaStream_t st)
{
    const int nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    const int nz = DIM == 3 ? L.nz : 1;
    const double* su = nullptr;
    const double* sl = nullptr;
    if (DIM == 3) {
        cudaError_t e = launch_kmv_sums(L, u, Tv, cl, bt, scratch, st);
        if (e == cudaSuccess) e = launch_kmv_sums(L, lam, Tv, cl, bt, scratch + (int64_t)bt.nsys * L.N * 4, st);
        if (e != cudaSuccess) return e;
        su = scratch;
        sl = scratch + (int64_t)bt.nsys * L.N * 4;
    }
    (void)Kn;
    return per_system<DIM>(nb, L, nset, st, [&](dim3 g, dim3 b, int s0) {
        k_grad<DIM, NB, DIM == 2><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, nset, u, lam, bt, su, sl, gKn, gTv, acc,
                                                   s0);
    });
}

}  // namespace

cudaError_t launch_stress(const Lattice& L, const double* u, const double* Kn, const double* Tv, const CoefLayout& cl,
                          const Batch& bt, const double* l0, double V, double* sig, double* scratch, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_stress<3>(TableNb<3>{L.nbr}, L, u, Kn, Tv, cl, bt, l0, V, sig, scratch, st);
        return run_stress<3>(GridNb<3>{L.nx, L.ny, L.nz}, L, u, Kn, Tv, cl, bt, l0, V, sig, scratch, st);
    }
    if (L.nbr) return run_stress<2>(TableNb<2>{L.nbr}, L, u, Kn, Tv, cl, bt, l0, V, sig, scratch, st);
    return run_stress<2>(GridNb<2>{L.nx, L.ny, 1}, L, u, Kn, Tv, cl, bt, l0, V, sig, scratch, st);
}

cudaError_t launch_energy(const Lattice& L, const double* u, const double* Kn, const double* Tv, const CoefLayout& cl,
                          const Batch& bt, double* w, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_energy<3>(TableNb<3>{L.nbr}, L, u, Kn, Tv, cl, bt, w, st);
        return run_energy<3>(GridNb<3>{L.nx, L.ny, L.nz}, L, u, Kn, Tv, cl, bt, w, st);
    }
    if (L.nbr) return run_energy<2>(TableNb<2>{L.nbr}, L, u, Kn, Tv, cl, bt, w, st);
    return run_energy<2>(GridNb<2>{L.nx, L.ny, 1}, L, u, Kn, Tv, cl, bt, w, st);
}

cudaError_t launch_grad(const Lattice& L, const double* u, const double* lam, const double* Kn, const double* Tv,
                        const CoefLayout& cl, const Batch& bt, double* gKn, double* gTv, double* scratch,
                        int accumulate, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_grad<3>(TableNb<3>{L.nbr}, L, u, lam, Kn, Tv, cl, bt, gKn, gTv, scratch, accumulate, st);
        return run_grad<3>(GridNb<3>{L.nx, L.ny, L.nz}, L, u, lam, Kn, Tv, cl, bt, gKn, gTv, scratch, accumulate, st);
    }
    if (L.nbr) return run_grad<2>(TableNb<2>{L.nbr}, L, u, lam, Kn, Tv, cl, bt, gKn, gTv, scratch, accumulate, st);
    return run_grad<2>(GridNb<2>{L.nx, L.ny, 1}, L, u, lam, Kn, Tv, cl, bt, gKn, gTv, scratch, accumulate, st);
}

template <typename T>
cudaError_t launch_pack(const double* src, T* dst, int64_t N, int NN, int nset, cudaStream_t st)
{
    for (int c0 = 0; c0 < nset; c0 += 65535) {
        const int nc = nset - c0 < 65535 ? nset - c0 : 65535;
        const dim3 g((unsigned)((N + 255) / 256), nc);
        k_pack<T><<<g, 256, 0, st>>>(src + (int64_t)c0 * N * NN, dst + (int64_t)c0 * N * NN, N, NN);
    }
    return cudaGetLastError();
}

template cudaError_t launch_pack<float>(const double*, float*, int64_t, int, int, cudaStream_t);
template cudaError_t launch_pack<double>(const double*, double*, int64_t, int, int, cudaStream_t);

cudaError_t launch_solid_nbr(int dim, int nx, int ny, int nz, int nspec, const uint8_t* solid, int32_t* nbr,
                             cudaStream_t st)
{
    const int64_t n = (int64_t)nx * ny * nz;
    const unsigned g = (unsigned)((n + 255) / 256);
    if (g == 0 || nspec < 1) return cudaSuccess;
    if (dim == 3)
        k_solid_nbr<3><<<dim3(g, nspec), 256, 0, st>>>(nx, ny, nz, solid, nbr);
    else
        k_solid_nbr<2><<<dim3(g, nspec), 256, 0, st>>>(nx, ny, 1, solid, nbr);
    return cudaGetLastError();
}

cudaError_t launch_build_nbr(int dim, int nx, int ny, int nz, int64_t n, const int64_t* site_of, const int64_t* sites,
                             int64_t* nbr, cudaStream_t st)
{
    const unsigned g = (unsigned)((n + 255) / 256);
    if (g == 0) return cudaSuccess;
    if (dim == 3)
        k_build_nbr<3><<<g, 256, 0, st>>>(nx, ny, nz, n, site_of, sites, nbr);
    else
        k_build_nbr<2><<<g, 256, 0, st>>>(nx, ny, 1, n, site_of, sites, nbr);
    return cudaGetLastError();
}

}  // namespace lpm
