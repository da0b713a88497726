// Matrix-free LPM operator K.u for the simple-cubic (3D, 18 slots) and square (2D, 8 slots) lattices.
//
// Two-pass form, batched over systems (right-hand sides) that share coefficient sets:
//   pass 1: per particle i and shell c:  S_i^c = sum_{k in c} dL_ik,  TS_i^c = sum_{k in c} Tv_ik dL_ik
//   pass 2 (SC, code-force form of coarse3d/lin3d.py:126-149):
//       F_ik = 2 Kn_ik dL_ik + (TS_i^c + TS_q^c)/2 + Tv_ik (S_i^c + S_q^c)/2,     f_i = sum_k F_ik n_k
//   pass 2 (SQ, exact-Hessian g-form of timing/t2d/solver2d.py:269-305):
//       g_ik = Kn_ik dL_ik + (Tv_ik S_i^c + TS_i^c)/2,  f_i = sum_k (g_ik + g_{q,k^1}) n_k
//     evaluated from the per-particle sums of q (no per-bond scratch): g_{q,k^1} needs Kn/Tv of q's slot k^1.
// The optional CG epilogue masks the result with the per-DOF free mask and reduces in . out per system with a
// deterministic last-block reduction.
//
// Structured boxes use implicit neighbours (site id (z*ny + y)*nx + x); other lattices (active-site masks) use an
// int32 neighbour table.  The fused single-pass z-marching SC kernel for full boxes lives in kmv_fused.cu.
#include "lpm_kernels.h"
#include "lpm_sqtile.cuh"
#include <atomic>
#include "lpm_stencil.cuh"

namespace lpm {

namespace {

using namespace stencil;

// ------------------------------------------------------------------------------------------------------ pass 1
template <typename T, int DIM, class NB>
__global__ void __launch_bounds__(256) k_shell_sums(NB nb, int nx, int ny, int nz, int64_t N, int sys0,
                                                    const T* __restrict__ u, const T* __restrict__ Tv, CoefLayout cl,
                                                    Batch bt, T* __restrict__ st, const int* __restrict__ act)
{
    const Site p = locate<NB>(nx, ny, nz, N, sys0);
    if (!p.ok || (act && !act[p.s])) return;
    const T* us = u + (int64_t)p.s * N * DIM;
    const T* tv = Tv + (int64_t)(p.s / bt.rhs_per_set) * cl.set_stride + p.i * cl.site_stride;
    T ui[3];
#pragma unroll
    for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
    auto load = [&](int64_t q, T* uq) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) uq[a] = us[DIM * q + a];
    };
    T v[4];
    shell_sums_at<T, DIM>(nb, p, ui, load, tv, cl.slot_stride, v);
    T* o = st + ((int64_t)p.s * N + p.i) * 4;
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
    o[3] = v[3];
}

// ------------------------------------------------------------------------------------------------------ pass 2
template <typename T, int DIM, class NB, bool EPI>
__global__ void __launch_bounds__(256) k_apply(NB nb, int nx, int ny, int nz, int64_t N, int sys0,
                                               const T* __restrict__ u, const T* __restrict__ Kn,
                                               const T* __restrict__ Tv, CoefLayout cl, Batch bt,
                                               const T* __restrict__ st, T* __restrict__ out,
                                               const uint8_t* __restrict__ mask, double* __restrict__ part,
                                               double* __restrict__ dot_final, unsigned* __restrict__ counter,
                                               const int* __restrict__ act, int nblk)
{
    const Site p = locate<NB>(nx, ny, nz, N, sys0);
    double dot = 0.0;
    if (p.ok && (!act || act[p.s])) {
        const T* us = u + (int64_t)p.s * N * DIM;
        const int64_t cbase = (int64_t)(p.s / bt.rhs_per_set) * cl.set_stride;
        const T* kn = Kn + cbase + p.i * cl.site_stride;
        const T* tv = Tv + cbase + p.i * cl.site_stride;
        const T* sts = st + (int64_t)p.s * N * 4;
        T ui[3];
#pragma unroll
        for (int a = 0; a < DIM; ++a) ui[a] = us[DIM * p.i + a];
        T Si[2], TSi[2];
        load4(sts + 4 * p.i, Si[0], Si[1], TSi[0], TSi[1]);
        auto load = [&](int64_t q, T* uq) {
#pragma unroll
            for (int a = 0; a < DIM; ++a) uq[a] = us[DIM * q + a];
        };
        auto sums = [&](int64_t q, T (&Sq)[2], T (&TSq)[2]) { load4(sts + 4 * q, Sq[0], Sq[1], TSq[0], TSq[1]); };
        T f[3];
        force_at<T, DIM>(nb, p, ui, load, sums, Si, TSi, kn, tv, Kn + cbase, Tv + cbase, cl, f);
        T* o = out + ((int64_t)p.s * N + p.i) * DIM;
        if (EPI && mask) {
            const uint8_t* m = mask + ((int64_t)(p.s % bt.nmask) * N + p.i) * DIM;
#pragma unroll
            for (int a = 0; a < DIM; ++a) f[a] = m[a] ? f[a] : T(0);
        }
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            o[a] = f[a];
            dot += (double)ui[a] * (double)f[a];
        }
    }
    if constexpr (EPI) {
        if (part == nullptr) return;
        __shared__ double sh[32];
        __shared__ bool last;
        const int tid = threadIdx.x + threadIdx.y * blockDim.x;
        const int nthr = blockDim.x * blockDim.y;
        const double v = block_sum(dot, sh);
        const int s = NB::structured ? sys0 + blockIdx.z / nz : sys0 + blockIdx.y;
        const int b = block_in_system<NB>(nz);
        if (tid == 0) {
            part[(int64_t)s * nblk + b] = v;
            __threadfence();
            last = atomicAdd(counter + s, 1u) == (unsigned)(nblk - 1);
        }
        __syncthreads();
        if (last) {
            double acc = 0.0;
            for (int j = tid; j < nblk; j += nthr) acc += __ldcg(part + (int64_t)s * nblk + j);
            acc = block_sum(acc, sh);
            if (tid == 0) {
                dot_final[s] = acc;
                counter[s] = 0u;
            }
        }
    }
}

// Kernel-side view of the fused CG p-update of MvEpilogue.
template <typename T>
struct PUpdate {
    const T* z;
    T* p0;  // read as the previous p, written as p' (the other buffer) by the tile's own sites
    T* p1;
    const double* beta;
    const int* pk;
};

// Full 2D boxes: both passes in one kernel (lpm_sqtile.cuh), one 32 x 8 tile of one system per block.  SC: the
// tile's Kn and Tv (tile + ring) are staged in shared memory with the displacements, in one phase with coalesced
// reads, and the shell sums and forces read no global memory; taken for the reference layout, whose per-site slot
// runs make the direct per-slot reads of a warp touch one sector per lane.  Without SC (packed layout, where a warp's
// per-slot reads are contiguous) the coefficients are read from global memory / L1 in the passes, which keeps the
// block at 18 KB of shared memory (FP64) and the SM at five blocks.  The optional epilogue masks the output and
// reduces u.out per system like k_apply (same block numbering).
template <typename T, bool EPI, bool SC, bool PF>
__global__ void __launch_bounds__(sqtile::NT) k_sq_fused(int nx, int ny, int64_t N, int sys0, const T* __restrict__ u,
                                                         const T* __restrict__ Kn, const T* __restrict__ Tv,
                                                         CoefLayout cl, Batch bt, T* __restrict__ out,
                                                         const uint8_t* __restrict__ mask, double* __restrict__ part,
                                                         double* __restrict__ dot_final,
                                                         unsigned* __restrict__ counter, const int* __restrict__ act,
                                                         PUpdate<T> pu)
{
    extern __shared__ __align__(16) unsigned char sq_dyn[];
    __shared__ std::conditional_t<SC, char, sqtile::Smem<T>> sm_static;
    sqtile::CoefSmem<T>& cs = *reinterpret_cast<sqtile::CoefSmem<T>*>(sq_dyn);
    sqtile::Smem<T>& sm = *[&]() {
        if constexpr (SC) return &cs.t;
        else return &sm_static;
    }();
    const int s = sys0 + blockIdx.z;
    if (act && !act[s]) return;
    const int x0 = blockIdx.x * sqtile::TX, y0 = blockIdx.y * sqtile::TY;
    const int64_t cbase = (int64_t)(s / bt.rhs_per_set) * cl.set_stride;
    // PF: p' = z + beta p from the previous p buffer; p' of the own sites goes to the other one
    const bool odd = PF && (pu.pk[s] & 1);
    const T* us = PF ? (odd ? pu.p1 : pu.p0) + (int64_t)s * N * 2 : u + (int64_t)s * N * 2;
    const T* zs = PF ? pu.z + (int64_t)s * N * 2 : nullptr;
    T* pn = PF ? (odd ? pu.p0 : pu.p1) + (int64_t)s * N * 2 : nullptr;
    const T be = PF ? (T)pu.beta[s] : T(0);
    auto load = [&](int64_t q, T* v) {
        if constexpr (PF) {
            v[0] = zs[2 * q] + be * us[2 * q];
            v[1] = zs[2 * q + 1] + be * us[2 * q + 1];
        } else {
            v[0] = us[2 * q];
            v[1] = us[2 * q + 1];
        }
    };
    using KA = std::conditional_t<SC, sqtile::SharedCoef<T>, sqtile::SoaCoef<T>>;
    KA kn, tv;
    if constexpr (SC) {
        sqtile::stage(nx, ny, x0, y0, load, sm);
        sqtile::stage_coef(nx, ny, x0, y0, Tv + cbase, cl, cs.tv);
        sqtile::stage_coef(nx, ny, x0, y0, Kn + cbase, cl, cs.kn);
        kn = KA{cs.kn};
        tv = KA{cs.tv};
    } else {
        sqtile::stage(nx, ny, x0, y0, load, sm);
        kn = KA(Kn + cbase, cl.slot_stride, nx, x0, y0);
        tv = KA(Tv + cbase, cl.slot_stride, nx, x0, y0);
    }
    __syncthreads();
    sqtile::sums(nx, ny, x0, y0, tv, sm);
    __syncthreads();
    double dot = 0.0;
    sqtile::forces(nx, ny, x0, y0, kn, tv, sm, [&](int64_t i, T (&f)[2], const T* ui) {
        if (EPI && mask) {
            const uint8_t* m = mask + ((int64_t)(s % bt.nmask) * N + i) * 2;
            f[0] = m[0] ? f[0] : T(0);
            f[1] = m[1] ? f[1] : T(0);
        }
        T* o = out + ((int64_t)s * N + i) * 2;
        o[0] = f[0];
        o[1] = f[1];
        if constexpr (PF) {
            pn[2 * i] = ui[0];
            pn[2 * i + 1] = ui[1];
        }
        dot += (double)ui[0] * (double)f[0] + (double)ui[1] * (double)f[1];
    });
    if constexpr (EPI) {
        if (part == nullptr) return;
        __shared__ double sh[32];
        __shared__ bool last;
        const int nblk = gridDim.x * gridDim.y;
        const int b = blockIdx.x + gridDim.x * blockIdx.y;
        const double v = block_sum(dot, sh);
        if (threadIdx.x == 0) {
            part[(int64_t)s * nblk + b] = v;
            __threadfence();
            last = atomicAdd(counter + s, 1u) == (unsigned)(nblk - 1);
        }
        __syncthreads();
        if (last) {
            double acc = 0.0;
            for (int j = threadIdx.x; j < nblk; j += sqtile::NT) acc += __ldcg(part + (int64_t)s * nblk + j);
            acc = block_sum(acc, sh);
            if (threadIdx.x == 0) {
                dot_final[s] = acc;
                counter[s] = 0u;
            }
        }
    }
}

// Several systems sharing a coefficient set: one block per tile and set stages the tile's coefficients (tile + ring,
// both arrays) in shared memory once and applies the operator to every system of the set, two per pass (one staging
// of both systems' displacements, one barrier-separated shell-sum and force phase for the pair), so a set's
// coefficients cross L2 once per tile instead of once per system.  Same arithmetic, output, epilogue and block
// numbering as k_sq_fused.  (Splitting a set's systems over more blocks, each staging the coefficients again, was
// slower: 0.065 -> 0.091 ms for six systems on a 512^2 box.)
// PF: the fused CG p-update of k_sq_fused, per system of the set.
template <typename T, bool EPI, bool PF = false>
__global__ void __launch_bounds__(sqtile::NT) k_sq_multi(int nx, int ny, int64_t N, int set0, const T* __restrict__ u,
                                                         const T* __restrict__ Kn, const T* __restrict__ Tv,
                                                         CoefLayout cl, Batch bt, T* __restrict__ out,
                                                         const uint8_t* __restrict__ mask, double* __restrict__ part,
                                                         double* __restrict__ dot_final,
                                                         unsigned* __restrict__ counter, const int* __restrict__ act,
                                                         PUpdate<T> pu = PUpdate<T>{})
{
    constexpr int NC = 8 * sqtile::SH * sqtile::SW;
    __shared__ sqtile::Smem<T> sm[2];
    __shared__ T ck[NC], ct[NC];
    __shared__ double sh[32];
    __shared__ bool last;
    const int set = set0 + blockIdx.z;
    const int s0 = set * bt.rhs_per_set;
    const int ns = min(bt.rhs_per_set, bt.nsys - s0);
    bool any = false;
    for (int j = 0; j < ns; ++j) any = any || !act || act[s0 + j];
    if (!any) return;
    const int x0 = blockIdx.x * sqtile::TX, y0 = blockIdx.y * sqtile::TY;
    const int64_t cbase = (int64_t)set * cl.set_stride;
    sqtile::stage_coef(nx, ny, x0, y0, Kn + cbase, cl, ck);
    sqtile::stage_coef(nx, ny, x0, y0, Tv + cbase, cl, ct);
    const sqtile::SharedCoef<T> kn{ck}, tv{ct};
    const int nblk = gridDim.x * gridDim.y;
    const int b = blockIdx.x + gridDim.x * blockIdx.y;
    for (int j = 0; j < ns; j += 2) {
        const int sa[2] = {s0 + j, s0 + j + 1};
        const bool on[2] = {!act || act[sa[0]], j + 1 < ns && (!act || act[sa[1]])};
        if (!on[0] && !on[1]) continue;  // the same for every thread of the block
        __syncthreads();  // the coefficients are staged and the previous pass's tiles are no longer read
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (!on[h]) continue;
            if constexpr (PF) {
                const int64_t so = (int64_t)sa[h] * N * 2;
                const T* us = ((pu.pk[sa[h]] & 1) ? pu.p1 : pu.p0) + so;
                const T* zs = pu.z + so;
                const T be = (T)pu.beta[sa[h]];
                sqtile::stage(nx, ny, x0, y0,
                              [&](int64_t q, T* v) {
                                  v[0] = zs[2 * q] + be * us[2 * q];
                                  v[1] = zs[2 * q + 1] + be * us[2 * q + 1];
                              },
                              sm[h]);
            } else {
                const T* us = u + (int64_t)sa[h] * N * 2;
                sqtile::stage(nx, ny, x0, y0,
                              [&](int64_t q, T* v) {
                                  v[0] = us[2 * q];
                                  v[1] = us[2 * q + 1];
                              },
                              sm[h]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (on[h]) sqtile::sums(nx, ny, x0, y0, tv, sm[h]);
        __syncthreads();
        double dot[2] = {0.0, 0.0};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (!on[h]) continue;
            const int s = sa[h];
            T* pn = PF ? ((pu.pk[s] & 1) ? pu.p0 : pu.p1) + (int64_t)s * N * 2 : nullptr;
            sqtile::forces(nx, ny, x0, y0, kn, tv, sm[h], [&](int64_t i, T (&f)[2], const T* ui) {
                if (EPI && mask) {
                    const uint8_t* m = mask + ((int64_t)(s % bt.nmask) * N + i) * 2;
                    f[0] = m[0] ? f[0] : T(0);
                    f[1] = m[1] ? f[1] : T(0);
                }
                T* o = out + ((int64_t)s * N + i) * 2;
                o[0] = f[0];
                o[1] = f[1];
                if constexpr (PF) {
                    pn[2 * i] = ui[0];
                    pn[2 * i + 1] = ui[1];
                }
                dot[h] += (double)ui[0] * (double)f[0] + (double)ui[1] * (double)f[1];
            });
        }
        if constexpr (EPI) {
            if (part == nullptr) continue;
            for (int h = 0; h < 2; ++h) {
                if (!on[h]) continue;
                const int s = sa[h];
                const double v = block_sum(dot[h], sh);
                if (threadIdx.x == 0) {
                    part[(int64_t)s * nblk + b] = v;
                    __threadfence();
                    last = atomicAdd(counter + s, 1u) == (unsigned)(nblk - 1);
                }
                __syncthreads();
                if (last) {
                    double acc = 0.0;
                    for (int q = threadIdx.x; q < nblk; q += sqtile::NT) acc += __ldcg(part + (int64_t)s * nblk + q);
                    acc = block_sum(acc, sh);
                    if (threadIdx.x == 0) {
                        dot_final[s] = acc;
                        counter[s] = 0u;
                    }
                }
                __syncthreads();  // `last` and `sh` are reused by the next system
            }
        }
    }
}

template <typename T>
cudaError_t run_sq_multi(const Lattice& L, const T* u, const T* Kn, const T* Tv, const CoefLayout& cl,
                         const Batch& bt, T* out, const MvEpilogue* ep, cudaStream_t st)
{
    const bool epi = ep && (ep->mask || ep->dot_part);
    const int* act = ep ? ep->act : nullptr;
    const bool pf = ep && ep->pz;
    if (pf && !epi) return cudaErrorInvalidValue;
    const int nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    for (int c0 = 0; c0 < nset; c0 += 65535) {
        const dim3 g(sqtile::tiles_x(L.nx), sqtile::tiles_y(L.ny), nset - c0 < 65535 ? nset - c0 : 65535);
        if (pf) {
            PUpdate<T> pu{static_cast<const T*>(ep->pz), static_cast<T*>(ep->p0), static_cast<T*>(ep->p1), ep->beta,
                          ep->pk};
            k_sq_multi<T, true, true><<<g, sqtile::NT, 0, st>>>(L.nx, L.ny, L.N, c0, u, Kn, Tv, cl, bt, out,
                                                                ep->mask, ep->dot_part, ep->dot_final, ep->counter,
                                                                act, pu);
        } else if (epi)
            k_sq_multi<T, true><<<g, sqtile::NT, 0, st>>>(L.nx, L.ny, L.N, c0, u, Kn, Tv, cl, bt, out, ep->mask,
                                                          ep->dot_part, ep->dot_final, ep->counter, act);
        else
            k_sq_multi<T, false><<<g, sqtile::NT, 0, st>>>(L.nx, L.ny, L.N, c0, u, Kn, Tv, cl, bt, out, nullptr,
                                                           nullptr, nullptr, nullptr, act);
    }
    return cudaGetLastError();
}

// Opt-in to k_sq_fused's dynamic shared memory (61 KB for FP64), once per device.
template <typename T, bool EPI, bool PF>
cudaError_t sq_fused_attr()  // the SC instantiation
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if ((done.load() >> dev) & 1ull) return cudaSuccess;
    e = cudaFuncSetAttribute(k_sq_fused<T, EPI, true, PF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(sqtile::CoefSmem<T>));
    if (e == cudaSuccess) done.fetch_or(1ull << dev);
    return e;
}

template <typename T>
cudaError_t run_sq_fused(const Lattice& L, const T* u, const T* Kn, const T* Tv, const CoefLayout& cl,
                         const Batch& bt, T* out, const MvEpilogue* ep, cudaStream_t st)
{
    // FP32 only: an FP64 tile's coefficients (43 KB) with its staging exceed the 48 KB of static shared memory
    if constexpr (sizeof(T) == 4) {
        if (bt.rhs_per_set > 1) return run_sq_multi<T>(L, u, Kn, Tv, cl, bt, out, ep, st);
    }
    const bool epi = ep && (ep->mask || ep->dot_part);
    const int* act = ep ? ep->act : nullptr;
    const bool sc = cl.site_stride != 1;  // all but the packed layout: coefficients staged in shared memory
    const bool pf = ep && ep->pz;
    if (pf && !epi) return cudaErrorInvalidValue;
    if (sc) {
        cudaError_t e = !epi ? sq_fused_attr<T, false, false>()
                             : (pf ? sq_fused_attr<T, true, true>() : sq_fused_attr<T, true, false>());
        if (e != cudaSuccess) return e;
    }
    const size_t smem = sc ? sizeof(sqtile::CoefSmem<T>) : 0;
    PUpdate<T> pu{};
    if (pf) {
        pu.z = static_cast<const T*>(ep->pz);
        pu.p0 = static_cast<T*>(ep->p0);
        pu.p1 = static_cast<T*>(ep->p1);
        pu.beta = ep->beta;
        pu.pk = ep->pk;
    }
    const dim3 grid(sqtile::tiles_x(L.nx), sqtile::tiles_y(L.ny), 1);
    for (int s0 = 0; s0 < bt.nsys; s0 += 65535) {
        dim3 g = grid;
        g.z = bt.nsys - s0 < 65535 ? bt.nsys - s0 : 65535;
        const uint8_t* mk = epi ? ep->mask : nullptr;
        double* dp = epi ? ep->dot_part : nullptr;
        double* df = epi ? ep->dot_final : nullptr;
        unsigned* ct = epi ? ep->counter : nullptr;
#define LPM_SQ_LAUNCH(E, S, P)                                                                                    \
    k_sq_fused<T, E, S, P><<<g, sqtile::NT, S ? smem : 0, st>>>(L.nx, L.ny, L.N, s0, u, Kn, Tv, cl, bt, out, mk, dp, \
                                                               df, ct, act, pu)
        if (!epi) {
            if (sc)
                LPM_SQ_LAUNCH(false, true, false);
            else
                LPM_SQ_LAUNCH(false, false, false);
        } else if (pf) {
            if (sc)
                LPM_SQ_LAUNCH(true, true, true);
            else
                LPM_SQ_LAUNCH(true, false, true);
        } else {
            if (sc)
                LPM_SQ_LAUNCH(true, true, false);
            else
                LPM_SQ_LAUNCH(true, false, false);
        }
#undef LPM_SQ_LAUNCH
    }
    return cudaGetLastError();
}

template <typename T, int DIM, class NB>
cudaError_t run_kmv(NB nb, const Lattice& L, const T* u, const T* Kn, const T* Tv, const CoefLayout& cl,
                    const Batch& bt, T* out, T* scratch, const MvEpilogue* ep, cudaStream_t st)
{
    if constexpr (DIM == 2 && NB::structured) return run_sq_fused<T>(L, u, Kn, Tv, cl, bt, out, ep, st);
    if (ep && ep->pz) return cudaErrorNotSupported;  // the fused p-update exists for full 2D boxes only
    const int nz = DIM == 3 ? L.nz : 1;
    const bool epi = ep && (ep->mask || ep->dot_part);  // act alone needs no epilogue
    int chunk, nblk;
    dim3 grid, block;
    if constexpr (NB::structured) {
        block = dim3(BX, BY, 1);
        chunk = 65535 / nz;
        grid = dim3((L.nx + BX - 1) / BX, (L.ny + BY - 1) / BY, 1);
        nblk = grid.x * grid.y * nz;
    } else {
        block = dim3(TB, 1, 1);
        chunk = 65535;
        grid = dim3((unsigned)((L.N + TB - 1) / TB), 1, 1);
        nblk = grid.x;
    }
    for (int s0 = 0; s0 < bt.nsys; s0 += chunk) {
        const int ns = bt.nsys - s0 < chunk ? bt.nsys - s0 : chunk;
        dim3 g = grid;
        if constexpr (NB::structured)
            g.z = nz * ns;
        else
            g.y = ns;
        const int* act = ep ? ep->act : nullptr;
        k_shell_sums<T, DIM, NB><<<g, block, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Tv, cl, bt, scratch, act);
        if (epi) {
            k_apply<T, DIM, NB, true><<<g, block, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Kn, Tv, cl, bt, scratch,
                                                           out, ep->mask, ep->dot_part, ep->dot_final, ep->counter,
                                                           act, nblk);
        } else {
            k_apply<T, DIM, NB, false><<<g, block, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Kn, Tv, cl, bt, scratch,
                                                            out, nullptr, nullptr, nullptr, nullptr, act, nblk);
        }
    }
    return cudaGetLastError();
}

}  // namespace

template <typename T, int DIM, class NB>
cudaError_t run_sums(NB nb, const Lattice& L, const T* u, const T* Tv, const CoefLayout& cl, const Batch& bt,
                     T* scratch, cudaStream_t st)
{
    const int nz = DIM == 3 ? L.nz : 1;
    int chunk;
    dim3 grid, block;
    if constexpr (NB::structured) {
        block = dim3(BX, BY, 1);
        chunk = 65535 / nz;
        grid = dim3((L.nx + BX - 1) / BX, (L.ny + BY - 1) / BY, 1);
    } else {
        block = dim3(TB, 1, 1);
        chunk = 65535;
        grid = dim3((unsigned)((L.N + TB - 1) / TB), 1, 1);
    }
    for (int s0 = 0; s0 < bt.nsys; s0 += chunk) {
        const int ns = bt.nsys - s0 < chunk ? bt.nsys - s0 : chunk;
        dim3 g = grid;
        if constexpr (NB::structured)
            g.z = nz * ns;
        else
            g.y = ns;
        k_shell_sums<T, DIM, NB><<<g, block, 0, st>>>(nb, L.nx, L.ny, nz, L.N, s0, u, Tv, cl, bt, scratch, nullptr);
    }
    return cudaGetLastError();
}

int kmv_dot_blocks(const Lattice& L)
{
    if (L.nbr) return (int)((L.N + TB - 1) / TB);
    if (L.dim == 2) return sqtile::tiles_x(L.nx) * sqtile::tiles_y(L.ny);
    const int nz = L.dim == 3 ? L.nz : 1;
    return ((L.nx + BX - 1) / BX) * ((L.ny + BY - 1) / BY) * nz;
}

template <typename T>
cudaError_t launch_kmv(const Lattice& L, const T* u, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                       T* out, T* scratch, const MvEpilogue* ep, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_kmv<T, 3>(TableNb<3>{L.nbr}, L, u, Kn, Tv, cl, bt, out, scratch, ep, st);
        return run_kmv<T, 3>(GridNb<3>{L.nx, L.ny, L.nz}, L, u, Kn, Tv, cl, bt, out, scratch, ep, st);
    }
    if (L.nbr) return run_kmv<T, 2>(TableNb<2>{L.nbr}, L, u, Kn, Tv, cl, bt, out, scratch, ep, st);
    return run_kmv<T, 2>(GridNb<2>{L.nx, L.ny, 1}, L, u, Kn, Tv, cl, bt, out, scratch, ep, st);
}

template <typename T>
cudaError_t launch_kmv_sums(const Lattice& L, const T* u, const T* Tv, const CoefLayout& cl, const Batch& bt,
                            T* scratch, cudaStream_t st)
{
    if (L.dim == 3) {
        if (L.nbr) return run_sums<T, 3>(TableNb<3>{L.nbr}, L, u, Tv, cl, bt, scratch, st);
        return run_sums<T, 3>(GridNb<3>{L.nx, L.ny, L.nz}, L, u, Tv, cl, bt, scratch, st);
    }
    if (L.nbr) return run_sums<T, 2>(TableNb<2>{L.nbr}, L, u, Tv, cl, bt, scratch, st);
    return run_sums<T, 2>(GridNb<2>{L.nx, L.ny, 1}, L, u, Tv, cl, bt, scratch, st);
}

template cudaError_t launch_kmv_sums<double>(const Lattice&, const double*, const double*, const CoefLayout&,
                                             const Batch&, double*, cudaStream_t);

template cudaError_t launch_kmv<float>(const Lattice&, const float*, const float*, const float*, const CoefLayout&,
                                       const Batch&, float*, float*, const MvEpilogue*, cudaStream_t);
template cudaError_t launch_kmv<double>(const Lattice&, const double*, const double*, const double*,
                                        const CoefLayout&, const Batch&, double*, double*, const MvEpilogue*,
                                        cudaStream_t);

}  // namespace lpm
