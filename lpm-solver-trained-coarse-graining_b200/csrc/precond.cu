// Block-Jacobi preconditioner: d x d diagonal blocks of K per particle and their inverses, per coefficient set.
//
//   D_p = sum_c 1/2 (T_c s_c^T + s_c T_c^T) + sum_{a valid} (Kn_pa + Kn_{q,a^1} + Tv_{q,a^1}) n_a n_a^T
//   T_c = sum_{a in c, valid} Tv_pa n_a,   s_c = sum_{a in c, valid} n_a
// (coarse3d/lin3d.py:239-269 k_block_diag; the 2D blocks of timing/t2d/solver2d.py:308-346 _diag_inv are the same
// expression with d = 2).  Inverses by cofactors as coarse3d/lin3d.py:272-291 (_inv3).  Built in FP64, stored in T.
#include "lpm_kernels.h"
#include "lpm_stencil.cuh"

namespace lpm {

namespace {

using namespace stencil;

template <typename T, int DIM, class NB>
__global__ void __launch_bounds__(256) k_block_jacobi(NB nb, int nx, int ny, int nz, int64_t N,
                                                      const double* __restrict__ Kn, const double* __restrict__ Tv,
                                                      CoefLayout cl, T* __restrict__ Minv, double* __restrict__ Dout,
                                                      int set0)
{
    using S = Slots<DIM>;
    const Site p = locate<NB>(nx, ny, nz, N, set0);  // p.s = coefficient set
    if (!p.ok) return;
    const int64_t cbase = (int64_t)p.s * cl.set_stride;
    double D[DIM][DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
        for (int b = 0; b < DIM; ++b) D[a][b] = 0.0;
    double Tc[2][DIM], sc[2][DIM];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int a = 0; a < DIM; ++a) Tc[c][a] = sc[c][a] = 0.0;
#pragma unroll
    for (int k = 0; k < S::NN; ++k) {
        int64_t q;
        if (!nb.get(p, k, q)) continue;
        const int c = S::shell(k);
        const double w = c == 0 ? 1.0 : INV_SQRT2;
        double n[3] = {-S::dx(k) * w, -S::dy(k) * w, -S::dz(k) * w};
        const double tvk = Tv[cbase + p.i * cl.site_stride + k * cl.slot_stride];
        const int64_t qo = cbase + q * cl.site_stride + (k ^ 1) * cl.slot_stride;
        const double coef = Kn[cbase + p.i * cl.site_stride + k * cl.slot_stride] + Kn[qo] + Tv[qo];
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            Tc[c][a] += tvk * n[a];
            sc[c][a] += n[a];
#pragma unroll
            for (int b = 0; b < DIM; ++b) D[a][b] += coef * n[a] * n[b];
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
            for (int b = 0; b < DIM; ++b) D[a][b] += 0.5 * (Tc[c][a] * sc[c][b] + sc[c][a] * Tc[c][b]);
    const int64_t o = ((int64_t)p.s * N + p.i) * DIM * DIM;
    if (Dout) {
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
            for (int b = 0; b < DIM; ++b) Dout[o + a * DIM + b] = D[a][b];
    }
    double M[DIM * DIM];
    if constexpr (DIM == 3) {
        const double a = D[0][0], b = D[0][1], c = D[0][2], d = D[1][0], e = D[1][1], f = D[1][2], g = D[2][0],
                     h = D[2][1], ii = D[2][2];
        const double co00 = e * ii - f * h, co01 = -(d * ii - f * g), co02 = d * h - e * g;
        const double det = a * co00 + b * co01 + c * co02;
        M[0] = co00 / det;
        M[3] = co01 / det;
        M[6] = co02 / det;
        M[1] = -(b * ii - c * h) / det;
        M[4] = (a * ii - c * g) / det;
        M[7] = -(a * h - b * g) / det;
        M[2] = (b * f - c * e) / det;
        M[5] = -(a * f - c * d) / det;
        M[8] = (a * e - b * d) / det;
    } else {
        const double det = D[0][0] * D[1][1] - D[0][1] * D[1][0];
        M[0] = D[1][1] / det;
        M[1] = -D[0][1] / det;
        M[2] = -D[1][0] / det;
        M[3] = D[0][0] / det;
    }
    // A particle without bonds (a void of a specimen with voids) has D = 0: its block is never used on a free DOF,
    // so store zero rather than 0/0, which would reach the engines' masked products as NaN * 0.
    bool finite = true;
#pragma unroll
    for (int a = 0; a < DIM * DIM; ++a) finite = finite && isfinite(M[a]);
#pragma unroll
    for (int a = 0; a < DIM * DIM; ++a) Minv[o + a] = finite ? (T)M[a] : T(0);
}

template <typename T, int DIM, class NB>
cudaError_t run_bj(NB nb, const Lattice& L, const double* Kn, const double* Tv, const CoefLayout& cl, int nset,
                   T* Minv, double* D, cudaStream_t st)
{
    const int nz = DIM == 3 ? L.nz : 1;
    if constexpr (NB::structured) {
        const int chunk = 65535 / nz;
        for (int s0 = 0; s0 < nset; s0 += chunk) {
            const int ns = nset - s0 < chunk ? nset - s0 : chunk;
            const dim3 g((L.nx + BX - 1) / BX, (L.ny + BY - 1) / BY, nz * ns);
            k_block_jacobi<T, DIM, NB><<<g, dim3(BX, BY), 0, st>>>(nb, L.nx, L.ny, nz, L.N, Kn, Tv, cl, Minv, D, s0);
        }
    } else {
        for (int s0 = 0; s0 < nset; s0 += 65535) {
            const int ns = nset - s0 < 65535 ? nset - s0 : 65535;
            const dim3 g((unsigned)((L.N + TB - 1) / TB), ns);
            k_block_jacobi<T, DIM, NB><<<g, TB, 0, st>>>(nb, L.nx, L.ny, nz, L.N, Kn, Tv, cl, Minv, D, s0);
        }
    }
    return cudaGetLastError();
}

}  // namespace

template <typename T>
cudaError_t launch_block_jacobi(const Lattice& L, const double* Kn, const double* Tv, const CoefLayout& cl, int nset,
                                T* Minv, double* D_out, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_bj<T, 3>(TableNb<3>{L.nbr}, L, Kn, Tv, cl, nset, Minv, D_out, st);
        return run_bj<T, 3>(GridNb<3>{L.nx, L.ny, L.nz}, L, Kn, Tv, cl, nset, Minv, D_out, st);
    }
    if (L.nbr) return run_bj<T, 2>(TableNb<2>{L.nbr}, L, Kn, Tv, cl, nset, Minv, D_out, st);
    return run_bj<T, 2>(GridNb<2>{L.nx, L.ny, 1}, L, Kn, Tv, cl, nset, Minv, D_out, st);
}

template cudaError_t launch_block_jacobi<float>(const Lattice&, const double*, const double*, const CoefLayout&, int,
                                                float*, double*, cudaStream_t);
template cudaError_t launch_block_jacobi<double>(const Lattice&, const double*, const double*, const CoefLayout&,
                                                 int, double*, double*, cudaStream_t);

}  // namespace lpm
