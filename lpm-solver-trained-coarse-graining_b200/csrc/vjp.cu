// Vector-Jacobian products of the post-processing outputs (FP64), for differentiable solves.
//
// Energy  U_i = 1/2 sum_k Kn dL^2 + 1/2 sum_c S_c TS_c, upstream weights G_i (per system):
//   dU_i/dKn_ik = 1/2 dL_ik^2,   dU_i/dTv_ik = 1/2 S_i^c dL_ik,
//   d(sum_i G_i U_i)/du_j = sum_k (G_j g_jk + G_q g_{q,k^1}) n_k,   g_ik = Kn dL + (Tv S_i^c + TS_i^c)/2
// (coarse3d/torch_lpm3d.py:89-92 energy, coarse2d/torch_lpm.py:252-258 energy_density, through autograd).
//
// Stress  sigma_i = sum_k a_ik F_ik n_k n_k^T, a_ik = of_ik l0_k / V (coarse3d/torch_lpm3d.py:85-87 stress,
// coarse2d/torch_lpm.py:246-250), upstream weights Gs_i (Voigt components).  With bond weights
// w_ik = a_ik (Gs_i . n_k n_k^T) the loss is sum_ik w_ik F_ik, F_ik the code-force bond force, and
//   dL/dKn_ik = 2 w_ik dL_ik,   dL/dTv_ik = 1/2 w_ik (S_i^c + S_q^c) + 1/2 dL_ik W_i^c,
//   dL/du_j   = sum_k (c_jk + c_{q,k^1}) n_k,   c_ik = 2 Kn_ik w_ik + 1/2 R_i^c + 1/2 Tv_ik W_i^c,
//   W_i^c = sum_{m in c} (w_im + w_{q_m,m^1}),  R_i^c = sum_{m in c} (Tv_im w_im + Tv_{q_m,m^1} w_{q_m,m^1}).
// Transpose product (the VJP of f = K u, coarse3d/torch_lpm3d.py:81-83 through autograd): the loss
// sum_i G_i . f_i = sum_ik (G_i . n_k) F_ik is the stress form with bond weights w_ik = G_i . n_k, so du = K^T G
// comes out of the same two passes; it differs from K G when the SC bond parameters are not symmetric.
// Parameter gradients are summed over the systems of each coefficient set (deterministically, one thread per
// particle and set).
#include "lpm_kernels.h"
#include "lpm_stencil.cuh"

namespace lpm {

namespace {

using namespace stencil;

// Site record of the neighbour q of p in slot k (grid coordinates only meaningful for structured lattices).
template <class NB>
__device__ __forceinline__ Site neighbour_site(const Site& p, int k, int64_t q)
{
    Site s = p;
    s.i = q;
    if constexpr (NB::structured) {
        constexpr int DIM = NB::dim;
        s.x = p.x + Slots<DIM>::dx(k);
        s.y = p.y + Slots<DIM>::dy(k);
        s.z = p.z + Slots<DIM>::dz(k);
    }
    return s;
}

template <int DIM, class NB>
__device__ __forceinline__ bool site_full(const NB& nb, const Site& p)
{
    bool full = true;
#pragma unroll
    for (int k = 0; k < Slots<DIM>::NN; ++k) {
        int64_t q;
        full = full && nb.get(p, k, q);
    }
    return full;
}

// Voigt weight of n_k n_k^T against G (3D: xx yy zz yz xz xy; 2D: xx yy xy).
template <int DIM>
__device__ __forceinline__ double voigt_w(const double* G, int k)
{
    using S = Slots<DIM>;
    const double w = S::shell(k) == 0 ? 1.0 : INV_SQRT2;
    const double n0 = -S::dx(k) * w, n1 = -S::dy(k) * w, n2 = -S::dz(k) * w;
    if constexpr (DIM == 3)
        return G[0] * n0 * n0 + G[1] * n1 * n1 + G[2] * n2 * n2 + G[3] * n1 * n2 + G[4] * n0 * n2 + G[5] * n0 * n1;
    else
        return G[0] * n0 * n0 + G[1] * n1 * n1 + G[2] * n0 * n1;
}

template <int DIM>
__device__ __forceinline__ void add_n(double* f, int k, double t)
{
    using S = Slots<DIM>;
    const double w = S::shell(k) == 0 ? 1.0 : INV_SQRT2;
    f[0] -= S::dx(k) * w * t;
    f[1] -= S::dy(k) * w * t;
    if constexpr (DIM == 3) f[2] -= S::dz(k) * w * t;
}

// ------------------------------------------------------------------------------------------------ energy VJP
template <int DIM, class NB>
__global__ void __launch_bounds__(256) k_energy_vjp(NB nb, int nx, int ny, int nz, int64_t N, int set0, Batch bt,
                                                    const double* __restrict__ u, const double* __restrict__ G,
                                                    const double* __restrict__ Kn, const double* __restrict__ Tv,
                                                    CoefLayout cl, const double* __restrict__ st,
                                                    double* __restrict__ du, double* __restrict__ gK,
                                                    double* __restrict__ gT, int acc)
{
    using S = Slots<DIM>;
    constexpr int NN = S::NN;
    const Site p = locate<NB>(nx, ny, nz, N, set0);
    if (!p.ok) return;
    const int set = p.s;
    const int s_lo = set * bt.rhs_per_set, s_hi = min(bt.nsys, s_lo + bt.rhs_per_set);
    const int64_t cb = (int64_t)set * cl.set_stride;
    double gk[NN], gt[NN];
#pragma unroll
    for (int k = 0; k < NN; ++k) gk[k] = gt[k] = 0.0;
    for (int s = s_lo; s < s_hi; ++s) {
        const double* us = u + (int64_t)s * N * DIM;
        const double* sts = st + (int64_t)s * N * 4;
        double ui[3];
#pragma unroll
        for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
        double Si[2], TSi[2];
        load4(sts + 4 * p.i, Si[0], Si[1], TSi[0], TSi[1]);
        const double Gi = G[(int64_t)s * N + p.i];
        double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < NN; ++k) {
            int64_t q;
            if (!nb.get(p, k, q)) continue;
            const int c = S::shell(k);
            const double d = dl_of<double, DIM>(us, p.i, q, k, ui);
            const int64_t io = cb + p.i * cl.site_stride + k * cl.slot_stride;
            const int64_t qo = cb + q * cl.site_stride + (k ^ 1) * cl.slot_stride;
            double Sq[2], TSq[2];
            load4(sts + 4 * q, Sq[0], Sq[1], TSq[0], TSq[1]);
            const double Gq = G[(int64_t)s * N + q];
            const double gi = Kn[io] * d + 0.5 * (Tv[io] * Si[c] + TSi[c]);
            const double gq = Kn[qo] * d + 0.5 * (Tv[qo] * Sq[c] + TSq[c]);
            add_n<DIM>(f, k, Gi * gi + Gq * gq);
            gk[k] += 0.5 * Gi * d * d;
            gt[k] += 0.5 * Gi * Si[c] * d;
        }
        double* o = du + ((int64_t)s * N + p.i) * DIM;
#pragma unroll
        for (int a = 0; a < DIM; ++a) o[a] = f[a];
    }
    double* ok = gK + ((int64_t)set * N + p.i) * NN;
    double* ot = gT + ((int64_t)set * N + p.i) * NN;
#pragma unroll
    for (int k = 0; k < NN; ++k) {
        ok[k] = acc ? ok[k] + gk[k] : gk[k];
        ot[k] = acc ? ot[k] + gt[k] : gt[k];
    }
}

// ------------------------------------------------------------------------------------------------ stress VJP
// MODE 1: stress weights a_ik (Gs_i . n_k n_k^T); MODE 2: transpose-product weights G_i . n_k.
template <int MODE, int DIM>
constexpr int weight_width() { return MODE == 2 ? DIM : (DIM == 3 ? 6 : 3); }

template <int MODE, int DIM, class NB>
__device__ __forceinline__ double bond_weight(const NB& nb, const Site& p, int k, bool full_p, const double* Gp,
                                              const double* l0, double V)
{
    if constexpr (MODE == 2) {
        double f[3] = {0.0, 0.0, 0.0};
        add_n<DIM>(f, k, 1.0);
        double w = Gp[0] * f[0] + Gp[1] * f[1];
        if constexpr (DIM == 3) w += Gp[2] * f[2];
        return w;
    } else {
        int64_t qq;
        const double of = (full_p || nb.get(p, k ^ 1, qq)) ? 0.5 : 1.0;
        return of / V * l0[k] * voigt_w<DIM>(Gp, k);
    }
}

template <int MODE, int DIM, class NB>
__device__ __forceinline__ bool site_full_if(const NB& nb, const Site& p)
{
    if constexpr (MODE == 2) return true;
    else return site_full<DIM>(nb, p);
}

// pass A: W^c and R^c of every particle and system -> wr (nsys, N, 4) = (W0, W1, R0, R1)
template <int MODE, int DIM, class NB>
__global__ void __launch_bounds__(256) k_stress_vjp_a(NB nb, int nx, int ny, int nz, int64_t N, int sys0, Batch bt,
                                                      const double* __restrict__ Gs, const double* __restrict__ Tv,
                                                      CoefLayout cl, const double* __restrict__ l0, double V,
                                                      double* __restrict__ wr)
{
    using S = Slots<DIM>;
    constexpr int NC = weight_width<MODE, DIM>();
    const Site p = locate<NB>(nx, ny, nz, N, sys0);
    if (!p.ok) return;
    const int s = p.s;
    const int64_t cb = (int64_t)(s / bt.rhs_per_set) * cl.set_stride;
    const double* Gp = Gs + ((int64_t)s * N + p.i) * NC;
    const bool full_p = site_full_if<MODE, DIM>(nb, p);
    double W[2] = {0.0, 0.0}, R[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        const int c = S::shell(k);
        const double wp = bond_weight<MODE, DIM>(nb, p, k, full_p, Gp, l0, V);
        const Site sq = neighbour_site<NB>(p, k, q);
        const double wq = bond_weight<MODE, DIM>(nb, sq, k ^ 1, site_full_if<MODE, DIM>(nb, sq),
                                                 Gs + ((int64_t)s * N + q) * NC, l0, V);
        W[c] += wp + wq;
        R[c] += Tv[cb + p.i * cl.site_stride + k * cl.slot_stride] * wp +
                Tv[cb + q * cl.site_stride + (k ^ 1) * cl.slot_stride] * wq;
    }
    double* o = wr + ((int64_t)s * N + p.i) * 4;
    o[0] = W[0];
    o[1] = W[1];
    o[2] = R[0];
    o[3] = R[1];
}

// pass B: du per system, parameter gradients per set
template <int MODE, int DIM, class NB>
__global__ void __launch_bounds__(256) k_stress_vjp_b(NB nb, int nx, int ny, int nz, int64_t N, int set0, Batch bt,
                                                      const double* __restrict__ u, const double* __restrict__ Gs,
                                                      const double* __restrict__ Kn, const double* __restrict__ Tv,
                                                      CoefLayout cl, const double* __restrict__ l0, double V,
                                                      const double* __restrict__ st, const double* __restrict__ wr,
                                                      double* __restrict__ du, double* __restrict__ gK,
                                                      double* __restrict__ gT, int acc)
{
    using S = Slots<DIM>;
    constexpr int NN = S::NN;
    constexpr int NC = weight_width<MODE, DIM>();
    const Site p = locate<NB>(nx, ny, nz, N, set0);
    if (!p.ok) return;
    const int set = p.s;
    const int s_lo = set * bt.rhs_per_set, s_hi = min(bt.nsys, s_lo + bt.rhs_per_set);
    const int64_t cb = (int64_t)set * cl.set_stride;
    const bool full_p = site_full_if<MODE, DIM>(nb, p);
    double gk[NN], gt[NN];
#pragma unroll
    for (int k = 0; k < NN; ++k) gk[k] = gt[k] = 0.0;
    for (int s = s_lo; s < s_hi; ++s) {
        const double* us = u + (int64_t)s * N * DIM;
        const double* sts = st + (int64_t)s * N * 4;
        const double* Gp = Gs + ((int64_t)s * N + p.i) * NC;
        double ui[3];
#pragma unroll
        for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
        double Si[2], TSi[2], Wi[2], Ri[2];
        load4(sts + 4 * p.i, Si[0], Si[1], TSi[0], TSi[1]);
        load4(wr + ((int64_t)s * N + p.i) * 4, Wi[0], Wi[1], Ri[0], Ri[1]);
        double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < NN; ++k) {
            int64_t q;
            if (!nb.get(p, k, q)) continue;
            const int c = S::shell(k);
            const double d = dl_of<double, DIM>(us, p.i, q, k, ui);
            const int64_t io = cb + p.i * cl.site_stride + k * cl.slot_stride;
            const int64_t qo = cb + q * cl.site_stride + (k ^ 1) * cl.slot_stride;
            const double wp = bond_weight<MODE, DIM>(nb, p, k, full_p, Gp, l0, V);
            const Site sq = neighbour_site<NB>(p, k, q);
            const double wq = bond_weight<MODE, DIM>(nb, sq, k ^ 1, site_full_if<MODE, DIM>(nb, sq),
                                                     Gs + ((int64_t)s * N + q) * NC, l0, V);
            double Sq[2], TSq[2], Wq[2], Rq[2];
            load4(sts + 4 * q, Sq[0], Sq[1], TSq[0], TSq[1]);
            load4(wr + ((int64_t)s * N + q) * 4, Wq[0], Wq[1], Rq[0], Rq[1]);
            const double ci = 2.0 * Kn[io] * wp + 0.5 * Ri[c] + 0.5 * Tv[io] * Wi[c];
            const double cq = 2.0 * Kn[qo] * wq + 0.5 * Rq[c] + 0.5 * Tv[qo] * Wq[c];
            add_n<DIM>(f, k, ci + cq);
            gk[k] += 2.0 * wp * d;
            gt[k] += 0.5 * wp * (Si[c] + Sq[c]) + 0.5 * d * Wi[c];
        }
        double* o = du + ((int64_t)s * N + p.i) * DIM;
#pragma unroll
        for (int a = 0; a < DIM; ++a) o[a] = f[a];
    }
    double* ok = gK + ((int64_t)set * N + p.i) * NN;
    double* ot = gT + ((int64_t)set * N + p.i) * NN;
#pragma unroll
    for (int k = 0; k < NN; ++k) {
        ok[k] = acc ? ok[k] + gk[k] : gk[k];
        ot[k] = acc ? ot[k] + gt[k] : gt[k];
    }
}

template <int DIM, class NB, typename F>
void grid_launch(const Lattice& L, int count, F&& launch)
{
    const int nz = DIM == 3 ? L.nz : 1;
    if constexpr (NB::structured) {
        const int chunk = 65535 / nz;
        for (int s0 = 0; s0 < count; s0 += chunk) {
            const int ns = count - s0 < chunk ? count - s0 : chunk;
            launch(dim3((L.nx + BX - 1) / BX, (L.ny + BY - 1) / BY, nz * ns), dim3(BX, BY), s0);
        }
    } else {
        for (int s0 = 0; s0 < count; s0 += 65535) {
            const int ns = count - s0 < 65535 ? count - s0 : 65535;
            launch(dim3((unsigned)((L.N + TB - 1) / TB), ns), dim3(TB), s0);
        }
    }
}

template <int DIM, class NB>
cudaError_t run_vjp(NB nb, const Lattice& L, int which, const double* u, const double* G, const double* Kn,
                    const double* Tv, const CoefLayout& cl, const Batch& bt, const double* l0, double V, double* du,
                    double* gK, double* gT, double* scratch, int acc, cudaStream_t st)
{
    const int nz = DIM == 3 ? L.nz : 1;
    const int nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    cudaError_t e = launch_kmv_sums<double>(L, u, Tv, cl, bt, scratch, st);
    if (e != cudaSuccess) return e;
    double* wr = scratch + (int64_t)bt.nsys * L.N * 4;
    if (which == 0) {
        grid_launch<DIM, NB>(L, nset, [&](dim3 g, dim3 b, int s0) {
            k_energy_vjp<DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, bt, u, G, Kn, Tv, cl, scratch, du, gK,
                                                   gT, acc);
        });
    } else if (which == 1) {
        grid_launch<DIM, NB>(L, bt.nsys, [&](dim3 g, dim3 b, int s0) {
            k_stress_vjp_a<1, DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, bt, G, Tv, cl, l0, V, wr);
        });
        grid_launch<DIM, NB>(L, nset, [&](dim3 g, dim3 b, int s0) {
            k_stress_vjp_b<1, DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, bt, u, G, Kn, Tv, cl, l0, V,
                                                        scratch, wr, du, gK, gT, acc);
        });
    } else if constexpr (DIM == 3) {
        grid_launch<DIM, NB>(L, bt.nsys, [&](dim3 g, dim3 b, int s0) {
            k_stress_vjp_a<2, DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, bt, G, Tv, cl, l0, V, wr);
        });
        grid_launch<DIM, NB>(L, nset, [&](dim3 g, dim3 b, int s0) {
            k_stress_vjp_b<2, DIM, NB><<<g, b, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, bt, u, G, Kn, Tv, cl, l0, V,
                                                        scratch, wr, du, gK, gT, acc);
        });
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_post_vjp(const Lattice& L, int which, const double* u, const double* G, const double* Kn,
                            const double* Tv, const CoefLayout& cl, const Batch& bt, const double* l0, double V,
                            double* du, double* gK, double* gT, double* scratch, int acc, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_vjp<3>(TableNb<3>{L.nbr}, L, which, u, G, Kn, Tv, cl, bt, l0, V, du, gK, gT, scratch, acc, st);
        return run_vjp<3>(GridNb<3>{L.nx, L.ny, L.nz}, L, which, u, G, Kn, Tv, cl, bt, l0, V, du, gK, gT, scratch, acc,
                          st);
    }
    if (L.nbr) return run_vjp<2>(TableNb<2>{L.nbr}, L, which, u, G, Kn, Tv, cl, bt, l0, V, du, gK, gT, scratch, acc, st);
    return run_vjp<2>(GridNb<2>{L.nx, L.ny, 1}, L, which, u, G, Kn, Tv, cl, bt, l0, V, du, gK, gT, scratch, acc, st);
}

}  // namespace lpm
