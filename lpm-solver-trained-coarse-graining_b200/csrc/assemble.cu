// Bond-parameter assembly upstream of the 3D solve (coarse3d/train3d.py):
//
//  * the symmetric scatter of per-group bond values to the (B, N, 18) parameter arrays (train3d.Scatter,
//    train3d.py:77-97): value j of a group goes to slot k_j of particle p_j and to slot k_j ^ 1 of its neighbour q_j,
//    and its adjoint, which sums the two slots of every bond;
//  * the smallest eigenpair of every (particle, shell) group bond Hessian of the stability penalty
//    (train3d.group_penalty, train3d.py:119-137):
//        H = diag(kn) + (tv 1^T + 1 tv^T) / 2 on the valid slots of the shell, and 1e3 sc on the diagonal of the
//        missing ones (sc = the sample's mean |Kn|),
//    by cyclic Jacobi rotations on the 6 x 6 (shell 0) or 12 x 12 (shell 1) matrix held by one thread; the eigenvector
//    gives the derivative of the eigenvalue (dlam/dH = v v^T for a simple eigenvalue).
#include <cstdint>

#include "../../include/lpm_b200.h"
#include "lpm_kernels.h"

namespace lpm {

namespace {

__global__ void k_bond_scatter(int64_t n, int64_t nb, const int32_t* __restrict__ p, const int32_t* __restrict__ k,
                               const int32_t* __restrict__ q, const double* __restrict__ vals, double* __restrict__ out)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int64_t b = blockIdx.y;
    const double v = vals[b * nb + j];
    double* o = out + b * n * 18;
    o[(int64_t)p[j] * 18 + k[j]] = v;
    if (q[j] >= 0) o[(int64_t)q[j] * 18 + (k[j] ^ 1)] = v;
}

__global__ void k_bond_gather_sym(int64_t n, int64_t nb, const int32_t* __restrict__ p, const int32_t* __restrict__ k,
                                  const int32_t* __restrict__ q, const double* __restrict__ G, double* __restrict__ g)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int64_t b = blockIdx.y;
    const double* Gb = G + b * n * 18;
    double v = Gb[(int64_t)p[j] * 18 + k[j]];
    if (q[j] >= 0) v += Gb[(int64_t)q[j] * 18 + (k[j] ^ 1)];
    g[b * nb + j] = v;
}

// Grid offsets of the 18 slots (the order of coarse3d/geom3d.py:16-19), for loops over slots with a runtime index.
__constant__ int c_off[18][3] = {{1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},   {0, 0, -1},
                                 {1, 1, 0},  {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1},  {-1, 0, -1},
                                 {1, 0, -1}, {-1, 0, 1}, {0, 1, 1},  {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};

constexpr int EG = 32;  // groups (threads) per block of the eigen kernel

// One thread per (sample, particle): the group Hessian of `shell` (slots 0..5 or 6..17) of a full box, and its
// smallest eigenpair by cyclic Jacobi rotations.  Each thread's matrix A and eigenvector matrix V live in shared
// memory, element (a, c) of thread j at [(a * M + c) * EG + j], so the threads of a warp touch consecutive words.
template <int M>
__global__ void __launch_bounds__(EG) k_group_eig(int nx, int ny, int nz, int nspec, const double* __restrict__ Kn,
                                                  const double* __restrict__ Tv, const double* __restrict__ sc,
                                                  double* __restrict__ lam_out, double* __restrict__ vec_out)
{
    extern __shared__ double eig_smem[];
    double* A = eig_smem + threadIdx.x;             // A(a, c) = A[(a * M + c) * EG]
    double* V = eig_smem + M * M * EG + threadIdx.x;
    auto at = [&](double* X, int a, int c) -> double& { return X[(a * M + c) * EG]; };

    const int64_t N = (int64_t)nx * ny * nz;
    const int64_t t = (int64_t)blockIdx.x * EG + threadIdx.x;
    if (t >= N * nspec) return;
    const int64_t b = t / N, i = t % N;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((int64_t)nx * ny));
    const int k0 = M == 6 ? 0 : 6;
    const double big = 1e3 * sc[b];
    const double* kn = Kn + (b * N + i) * 18 + k0;
    const double* tv = Tv + (b * N + i) * 18 + k0;
    unsigned vmask = 0;
    for (int a = 0; a < M; ++a) {
        const int k = k0 + a;
        const int qx = x + c_off[k][0], qy = y + c_off[k][1], qz = z + c_off[k][2];
        if (qx >= 0 && qx < nx && qy >= 0 && qy < ny && qz >= 0 && qz < nz) vmask |= 1u << a;
    }
    double scale = 0.0;
    for (int a = 0; a < M; ++a) {
        const bool va = (vmask >> a) & 1u;
        for (int c = 0; c < M; ++c) {
            const bool vc = (vmask >> c) & 1u;
            double h = (va && vc) ? 0.5 * (tv[a] + tv[c]) : 0.0;
            if (a == c) h += va ? kn[a] : big;
            at(A, a, c) = h;
            at(V, a, c) = a == c ? 1.0 : 0.0;
            scale += h * h;
        }
    }
    for (int sweep = 0; sweep < 40; ++sweep) {
        double off = 0.0;
        for (int a = 0; a < M; ++a)
            for (int c = a + 1; c < M; ++c) off += at(A, a, c) * at(A, a, c);
        if (off <= 1e-32 * scale) break;
        for (int p = 0; p < M - 1; ++p) {
            for (int r = p + 1; r < M; ++r) {
                const double apr = at(A, p, r);
                if (apr == 0.0) continue;
                // the rotation in the (p, r) plane that zeroes A(p, r), tangent in its stable form
                const double theta = (at(A, r, r) - at(A, p, p)) / (2.0 * apr);
                const double tn = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(tn * tn + 1.0), sn = tn * cs;
                for (int m = 0; m < M; ++m) {  // columns p, r
                    const double amp = at(A, m, p), amr = at(A, m, r);
                    at(A, m, p) = cs * amp - sn * amr;
                    at(A, m, r) = sn * amp + cs * amr;
                }
                for (int m = 0; m < M; ++m) {  // rows p, r
                    const double apm = at(A, p, m), arm = at(A, r, m);
                    at(A, p, m) = cs * apm - sn * arm;
                    at(A, r, m) = sn * apm + cs * arm;
                }
                for (int m = 0; m < M; ++m) {
                    const double vmp = at(V, m, p), vmr = at(V, m, r);
                    at(V, m, p) = cs * vmp - sn * vmr;
                    at(V, m, r) = sn * vmp + cs * vmr;
                }
            }
        }
    }
    int im = 0;
    for (int a = 1; a < M; ++a)
        if (at(A, a, a) < at(A, im, im)) im = a;
    lam_out[t] = at(A, im, im);
    for (int a = 0; a < M; ++a) vec_out[t * M + a] = at(V, a, im);
}

}  // namespace

}  // namespace lpm

using namespace lpm;

int lpm_bond_scatter_f64(int32_t nspec, int64_t n, int64_t nb, const int32_t* p, const int32_t* k, const int32_t* q,
                         const double* vals, double* out, void* stream)
{
    if (nspec < 1 || nspec > 65535 || n < 1 || nb < 0 || (nb > 0 && (!p || !k || !q || !vals)) || !out)
        return LPM_ERR_ARG;
    if (nb == 0) return LPM_OK;
    k_bond_scatter<<<dim3((unsigned)((nb + 255) / 256), nspec), 256, 0, (cudaStream_t)stream>>>(n, nb, p, k, q, vals,
                                                                                                  out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LPM_OK : (int)e;
}

int lpm_bond_gather_sym_f64(int32_t nspec, int64_t n, int64_t nb, const int32_t* p, const int32_t* k,
                            const int32_t* q, const double* G, double* g, void* stream)
{
    if (nspec < 1 || nspec > 65535 || n < 1 || nb < 0 || (nb > 0 && (!p || !k || !q || !g)) || !G) return LPM_ERR_ARG;
    if (nb == 0) return LPM_OK;
    k_bond_gather_sym<<<dim3((unsigned)((nb + 255) / 256), nspec), 256, 0, (cudaStream_t)stream>>>(n, nb, p, k, q, G,
                                                                                                     g);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LPM_OK : (int)e;
}

int lpm_group_eigmin_sc(const lpm_lattice* lat, int32_t nspec, const double* Kn, const double* Tv, const double* sc,
                        int32_t shell, double* lam, double* vec, void* stream)
{
    if (!lat || lat->dim != 3 || lat->nbr || nspec < 1 || !Kn || !Tv || !sc || !lam || !vec ||
        (shell != 0 && shell != 1))
        return LPM_ERR_ARG;
    if ((int64_t)lat->nx * lat->ny * lat->nz != lat->n) return LPM_ERR_ARG;
    const int64_t tot = lat->n * nspec;
    const unsigned g = (unsigned)((tot + EG - 1) / EG);
    cudaStream_t st = (cudaStream_t)stream;
    if (shell == 0) {
        k_group_eig<6><<<g, EG, 2 * 36 * EG * sizeof(double), st>>>(lat->nx, lat->ny, lat->nz, nspec, Kn, Tv, sc, lam,
                                                                      vec);
    } else {
        constexpr int bytes = 2 * 144 * EG * sizeof(double);  // 73,728 B: above the 48 KB default, opted in once
        static unsigned long long attr_set = 0;  // devices on which the opt-in was made
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return (int)e;
        if (dev < 0 || dev >= 64) return LPM_ERR_UNSUPPORTED;
        if (!((attr_set >> dev) & 1ull)) {
            e = cudaFuncSetAttribute(k_group_eig<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e != cudaSuccess) return (int)e;
            attr_set |= 1ull << dev;
        }
        k_group_eig<12><<<g, EG, bytes, st>>>(lat->nx, lat->ny, lat->nz, nspec, Kn, Tv, sc, lam, vec);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LPM_OK : (int)e;
}
