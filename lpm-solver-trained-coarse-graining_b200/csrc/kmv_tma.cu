// TMA-fed fused SC operator for full boxes: out = K u (code-force form, coarse3d/lin3d.py:126-149), one kernel,
// batched over the right-hand sides that share a coefficient set.
//
// Decomposition (per particle i, shell c, A = TS/2, B = S/2, n_k = -w_k o_k, sums over existing bonds):
//   f_i  = own_i + sum_k n_k (A_q^c + Tv_ik B_q^c)
//   own_i = sum_k 2 Kn_ik dL_ik n_k + sum_c (A_i^c s_i^c + B_i^c T_i^c),  s_i^c = sum_{k in c} n_k,
//           T_i^c = sum_{k in c} Tv_ik n_k
// i.e. F_ik = 2 Kn dL + (TS_i + TS_q)/2 + Tv (S_i + S_q)/2 against n_k, regrouped so a particle's own terms are formed
// while its dL are in registers and only (B, A) of the neighbours is exchanged through shared memory.
//
// Tiling: a CTA owns a TX x TY column of the box, a range of z planes and NR systems of one coefficient set (FP32:
// up to 3, FP64: up to 2), and marches in z.  Step z: phase 1 on plane z+1 (shell sums of tile + 1-site ring, own terms of the tile), phase 2 on
// plane z (neighbour terms, output).  All global inputs arrive by TMA (cp.async.bulk.tensor, no multicast), issued by
// one thread a full step ahead into shared-memory rings guarded by mbarriers:
//   u  : 4 planes x NR systems x (TY+4) rows x 112 values (AoS x,y,z interleaved; x window x0-2 .. x0+33)
//   Tv : 2 planes x 18 slots x (TY+2) rows x 40 sites   (x window x0-4 .. x0+35)
//   Kn : 2 planes x 18 slots x TY rows x 32 sites
// (B, A) of 3 planes live in shared memory too.  Every mbarrier wait is bounded; on expiry the kernel records an
// error code, stops, and returns without touching its buffers further.
//
// Epilogue (EPI): out = mask(f), per-system u.out partials reduced deterministically; the last block of a system runs
// the CG alpha step.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <atomic>

#include <mutex>
#include <type_traits>

#include "lpm_fused.h"
#include "lpm_ptx.cuh"
#include "lpm_tma.h"

namespace lpm {

namespace {

using namespace ptx;

constexpr int TX = 32;
constexpr int UXW = 112;  // values per u row in the window (16-byte aligned start 3*x0 - 8)
constexpr int TVW = 40;   // sites per Tv row (start x0 - 4)

template <typename T>
struct T2;
template <>
struct T2<float> {
    using type = float2;
};
template <>
struct T2<double> {
    using type = double2;
};

template <typename T>
__device__ __forceinline__ T wk(int k)
{
    return sc_shell(k) == 0 ? T(1) : T(INV_SQRT2);
}

// Slot validity masks: bits of slots with dx = -1 / +1, dy = -1 / +1, dz = -1 / +1.
__host__ __device__ constexpr unsigned dir_mask(int axis, int sgn)
{
    unsigned m = 0;
    for (int k = 0; k < 18; ++k) {
        const int d = axis == 0 ? sc_dx(k) : axis == 1 ? sc_dy(k) : sc_dz(k);
        if (d == sgn) m |= 1u << k;
    }
    return m;
}

// Three extra warps (rows TY .. TY+2 of the block) take the halo-ring sites, so the tile warps carry none and the
// block barrier after phase 1 waits for no straggling ring work.
constexpr int RY = 3, RT = TX * RY;

template <typename T, int NR, int TY>
struct Layout {
    static constexpr int NT = TX * TY;          // tile threads
    static constexpr int NTH = TX * (TY + RY);  // all threads
    static constexpr int UH = TY + 4;
    static constexpr int SW = TX + 2, SH = TY + 2, SPL = SW * SH;
    static constexpr int NRING = SPL - NT;
    static constexpr size_t U_SLOT = (size_t)NR * UH * UXW * sizeof(T);
    static constexpr size_t TV_SLOT = (size_t)18 * SH * TVW * sizeof(T);
    static constexpr size_t KN_SLOT = (size_t)18 * TY * TX * sizeof(T);
    static constexpr size_t ST_SLOT = (size_t)NR * 2 * SPL * 2 * sizeof(T);
    static constexpr size_t OFF_TV = 4 * U_SLOT;
    static constexpr size_t OFF_KN = OFF_TV + 2 * TV_SLOT;
    static constexpr size_t OFF_ST = OFF_KN + 2 * KN_SLOT;
    static constexpr size_t BYTES = OFF_ST + 3 * ST_SLOT;
    static_assert(U_SLOT % 128 == 0 && TV_SLOT % 128 == 0 && KN_SLOT % 128 == 0, "TMA slots must stay 128B aligned");
};

template <typename T, int NR, int TY, bool EPI>
__global__ void __launch_bounds__(TX*(TY + RY), 1)
    k_sc_tma(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_tv,
             const __grid_constant__ CUtensorMap tm_kn, TmaArgs<T> P)
{
    using Lay = Layout<T, NR, TY>;
    using V2 = typename T2<T>::type;
    constexpr int NT = Lay::NT, NTH = Lay::NTH, UH = Lay::UH, SW = Lay::SW, SH = Lay::SH, SPL = Lay::SPL;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[8];  // u: 0..3, Tv: 4..5, Kn: 6..7
    __shared__ double red[32];
    __shared__ int abort_flag;
    __shared__ bool last_flag;

    T* su = reinterpret_cast<T*>(smem);
    T* stv = reinterpret_cast<T*>(smem + Lay::OFF_TV);
    T* skn = reinterpret_cast<T*>(smem + Lay::OFF_KN);
    V2* sst = reinterpret_cast<V2*>(smem + Lay::OFF_ST);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY;
    // Grid: x = (system group of the set, column tile, z chunk) with the group fastest, y = coefficient set: the groups
    // of a set run together and share the set's coefficient tiles through L2.
    const int g = blockIdx.x % P.ngrp, tz = blockIdx.x / P.ngrp;  // tz: this CTA's block index within its systems
    const int tile = tz % (ntx * nty), zc = tz / (ntx * nty);
    const int x0 = (tile % ntx) * TX, y0 = (tile / ntx) * TY;
    const int set = blockIdx.y + P.set0;
    const int sbase = set * P.rhs_per_set + g * NR;
    int nr = P.rhs_per_set - g * NR;
    nr = nr < NR ? nr : NR;
    if (sbase + nr > P.nsys) nr = P.nsys - sbase;
    const int zbeg = zc * P.zchunk;
    const int zend = min(nz, zbeg + P.zchunk);

    bool on[NR];
    bool any_on = false;
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        on[j] = j < nr && (!P.act || P.act[sbase + j]);
        any_on |= on[j];
    }

    if (tid == 0) {
        for (int b = 0; b < 8; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
        abort_flag = 0;
        // TMA destinations must be 128-byte aligned; refuse to run (and report) otherwise
        if (saddr(smem) & 127u) {
            abort_flag = 1;
            if (P.err) atomicExch(P.err, 2);
        }
    }
    {
        V2 zz;
        zz.x = zz.y = T(0);
        for (int e = tid; e < 3 * NR * 2 * SPL; e += NTH) sst[e] = zz;
        // u slots that will stand for planes below 0 are never loaded; they must read as finite values (zero),
        // because invalid bonds are removed by multiplying with 0
        const int nneg = zc * P.zchunk - 2 < 0 ? 2 - zc * P.zchunk : 0;  // planes zbeg-2 .. -1
        for (int e = tid; e < nneg * (int)(Lay::U_SLOT / sizeof(T)); e += NTH) su[e] = T(0);
    }
    __syncthreads();
    if (abort_flag) any_on = false;

    // ------------------------------------------------------------------------------------------- producer side
    // Plane fills are numbered from the first plane each stream loads; slot = n % nslots, parity = (n / nslots) & 1.
    const int u0 = zbeg - 2, tv0 = zbeg - 1, kn0 = zbeg;
    constexpr uint32_t U_BYTES = (uint32_t)(NR * UH * UXW * sizeof(T));
    constexpr uint32_t TV_BYTES = (uint32_t)(18 * SH * TVW * sizeof(T));
    constexpr uint32_t KN_BYTES = (uint32_t)(18 * TY * TX * sizeof(T));
    const int coef_plane0 = set * 18;  // 4th tensor coordinate of slot 0 of this set
    // Thread 0 keeps the parity of the last fill issued on each barrier (bit b of `ppar`, and bit b of `pend` while
    // it may still be in flight) so that an aborting block can let its copies land before it exits.
    unsigned pend = 0, ppar = 0;
    auto note = [&](int b, int parity) {
        pend |= 1u << b;
        ppar = (ppar & ~(1u << b)) | ((unsigned)parity << b);
    };
    auto issue_u = [&](int p) {
        const int n = p - u0;
        uint64_t* bar = &bars[n & 3];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, U_BYTES);
        tma_load4(su + (size_t)(n & 3) * (Lay::U_SLOT / sizeof(T)), &tm_u, bar, 3 * x0 - 8, y0 - 2, p, sbase);
        note(n & 3, (n >> 2) & 1);
    };
    auto issue_tv = [&](int p) {
        const int n = p - tv0;
        uint64_t* bar = &bars[4 + (n & 1)];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, TV_BYTES);
        tma_load4(stv + (size_t)(n & 1) * (Lay::TV_SLOT / sizeof(T)), &tm_tv, bar, x0 - 4, y0 - 1, p, coef_plane0);
        note(4 + (n & 1), (n >> 1) & 1);
    };
    auto issue_kn = [&](int p) {
        const int n = p - kn0;
        uint64_t* bar = &bars[6 + (n & 1)];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, KN_BYTES);
        tma_load4(skn + (size_t)(n & 1) * (Lay::KN_SLOT / sizeof(T)), &tm_kn, bar, x0, y0, p, coef_plane0);
        note(6 + (n & 1), (n >> 1) & 1);
    };
    // Thread 0 waits (bounded) for the listed in-range fills, then the block synchronises; every thread then
    // observes the completed phases itself (immediate) before reading.  The abort decision is the OR over the block
    // at that barrier (__syncthreads_or), so all threads return at the same step: a shared flag written by thread 0
    // could already hold the next step's expiry when a slow warp reads it.
    auto wait_planes = [&](int pu, int ptv, int pkn) -> bool {
        auto ok_u = [&](int p) { return p >= 0 && p < nz && p >= u0; };
        auto ok_tv = [&](int p) { return p >= 0 && p < nz && p >= tv0; };
        auto ok_kn = [&](int p) { return p >= 0 && p < nz && p >= kn0 && p < zend; };
        bool good = true;
        if (tid == 0) {
            const unsigned lim = P.wait_polls;
            if (ok_u(pu)) good = good && mbar_wait(&bars[(pu - u0) & 3], ((pu - u0) >> 2) & 1, lim);
            if (ok_tv(ptv)) good = good && mbar_wait(&bars[4 + ((ptv - tv0) & 1)], ((ptv - tv0) >> 1) & 1, lim);
            if (ok_kn(pkn)) good = good && mbar_wait(&bars[6 + ((pkn - kn0) & 1)], ((pkn - kn0) >> 1) & 1, lim);
            if (!good && P.err) atomicExch(P.err, 1);
        }
        if (__syncthreads_or(!good)) return false;
        if (ok_u(pu)) mbar_wait(&bars[(pu - u0) & 3], ((pu - u0) >> 2) & 1);
        if (ok_tv(ptv)) mbar_wait(&bars[4 + ((ptv - tv0) & 1)], ((ptv - tv0) >> 1) & 1);
        if (ok_kn(pkn)) mbar_wait(&bars[6 + ((pkn - kn0) & 1)], ((pkn - kn0) >> 1) & 1);
        return true;
    };

    // ---------------------------------------------------------------------------------------------- phase 1
    // Straight-line over the 18 slots: bond validity enters through selects (reads of out-of-box or not-loaded
    // values are in bounds of shared memory and are discarded by the select, whatever they hold).  Diagonal-slot
    // quantities are accumulated without the 1/sqrt2 factor and scaled once: dL = w d', 2 Kn w dL = Kn d' (w^2 = 1/2).
    // Shell-1 (B, A) are stored pre-multiplied by w for phase 2.
    T own_next[NR][3];
    T tv_next[18];
    auto u_slot = [&](int p) { return su + (size_t)((p - u0) & 3) * (Lay::U_SLOT / sizeof(T)); };
    auto tv_slot = [&](int p) { return stv + (size_t)((p - tv0) & 1) * (Lay::TV_SLOT / sizeof(T)); };
    auto kn_slot = [&](int p) { return skn + (size_t)((p - kn0) & 1) * (Lay::KN_SLOT / sizeof(T)); };
    auto st_slot = [&](int p) { return sst + (size_t)(((p % 3) + 3) % 3) * (Lay::ST_SLOT / sizeof(V2)); };
    const T W = T(INV_SQRT2);
    // (B, A) of a plane outside the box is zero, so that phase 2 needs no validity test (planes -1 and nz)
    auto zero_st = [&](int zp) {
        V2* dst = st_slot(zp);
        V2 zz;
        zz.x = zz.y = T(0);
        for (int e = tid; e < NR * 2 * SPL; e += NTH) dst[e] = zz;
    };

    // shell sums (and own terms) of system j at site (qx, qy) of plane zp, given the site's Tv and validity
    auto site_sys = [&](int j, int qx, int qy, int zp, const T* vk, const T* tv, const T* knw, auto own_tag,
                        const T (*sc)[3], const T (*Tc)[3]) {
        constexpr bool OWN = decltype(own_tag)::value;
        const T* pm = u_slot(zp - 1) + j * UH * UXW;
        const T* p0 = u_slot(zp) + j * UH * UXW;
        const T* pp = u_slot(zp + 1) + j * UH * UXW;
        const int ux = qx + 1, uy = qy + 1;
        const int ci = uy * UXW + 3 * ux + 2;
        const T ui[3] = {p0[ci], p0[ci + 1], p0[ci + 2]};
        T d[18];
#pragma unroll
        for (int k = 0; k < 18; ++k) {
            const T* pl = sc_dz(k) < 0 ? pm : (sc_dz(k) > 0 ? pp : p0);
            const int qo = ci + sc_dy(k) * UXW + 3 * sc_dx(k);
            T v = T(0);
            if (sc_dx(k)) v += T(sc_dx(k)) * (pl[qo] - ui[0]);
            if (sc_dy(k)) v += T(sc_dy(k)) * (pl[qo + 1] - ui[1]);
            if (sc_dz(k)) v += T(sc_dz(k)) * (pl[qo + 2] - ui[2]);
            d[k] = vk[k] * v;
        }
        T S0 = (d[0] + d[1]) + (d[2] + d[3]) + (d[4] + d[5]);
        T S1 = ((d[6] + d[7]) + (d[8] + d[9])) + ((d[10] + d[11]) + (d[12] + d[13])) + ((d[14] + d[15]) + (d[16] + d[17]));
        T TS0 = T(0), TS1a = T(0), TS1b = T(0);
#pragma unroll
        for (int k = 0; k < 6; ++k) TS0 += tv[k] * d[k];
#pragma unroll
        for (int k = 6; k < 12; ++k) TS1a += tv[k] * d[k];
#pragma unroll
        for (int k = 12; k < 18; ++k) TS1b += tv[k] * d[k];
        S1 *= W;
        const T TS1 = (TS1a + TS1b) * W;
        V2* dst = st_slot(zp) + j * 2 * SPL + qy * SW + qx;
        V2 v0, v1;
        v0.x = T(0.5) * S0;
        v0.y = T(0.5) * TS0;
        v1.x = T(0.5) * W * S1;
        v1.y = T(0.5) * W * TS1;
        dst[0] = v0;
        dst[SPL] = v1;
        if constexpr (OWN) {
            T f[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int k = 0; k < 18; ++k) {
                const T kd = knw[k] * d[k];
                if (sc_dx(k)) f[0] -= T(sc_dx(k)) * kd;
                if (sc_dy(k)) f[1] -= T(sc_dy(k)) * kd;
                if (sc_dz(k)) f[2] -= T(sc_dz(k)) * kd;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a)
                own_next[j][a] = f[a] + T(0.5) * (TS0 * sc[0][a] + S0 * Tc[0][a] + TS1 * sc[1][a] + S1 * Tc[1][a]);
        }
    };

    // masks of the slots that leave the box through each face
    constexpr unsigned XN = dir_mask(0, -1), XP = dir_mask(0, 1), YN = dir_mask(1, -1), YP = dir_mask(1, 1),
                       ZN = dir_mask(2, -1), ZP = dir_mask(2, 1);
    auto xy_mask = [&](int X, int Y) {
        unsigned m = 0x3FFFFu;
        if (X == 0) m &= ~XN;
        if (X == nx - 1) m &= ~XP;
        if (Y == 0) m &= ~YN;
        if (Y == ny - 1) m &= ~YP;
        return m;
    };
    auto z_mask = [&](int z) {
        unsigned m = 0x3FFFFu;
        if (z == 0) m &= ~ZN;
        if (z == nz - 1) m &= ~ZP;
        return m;
    };

    const int gx = x0 + tx, gy = y0 + ty;
    const bool own_xy = ty < TY && gx < nx && gy < ny;
    const unsigned own_mxy = xy_mask(gx, gy);
    // halo-ring work items of the ring threads (tid >= NT): item e = (tid - NT) + it * RT (it < NIT) is ring site
    // e % NRING of system e / NRING; the first is resolved once, later ones in every z step (fewer live registers).
    constexpr int NITEM = Lay::NRING * NR;
    constexpr int NIT = (NITEM + RT - 1) / RT;
    struct RingItem {
        int rj, rqx, rqy;
        bool in;
        unsigned mxy;
    };
    auto ring_item = [&](int it) {
        const int e = (tid - NT) + it * RT;
        const bool has_item = tid >= NT && e < NITEM;
        const int rs = has_item ? e % Lay::NRING : 0, rj = has_item ? e / Lay::NRING : 0;
        int rqx, rqy;
        if (rs < SW) {
            rqx = rs;
            rqy = 0;
        } else if (rs < 2 * SW) {
            rqx = rs - SW;
            rqy = SH - 1;
        } else if (rs < 2 * SW + TY) {
            rqx = 0;
            rqy = rs - 2 * SW + 1;
        } else {
            rqx = SW - 1;
            rqy = rs - 2 * SW - TY + 1;
        }
        const int rX = x0 - 1 + rqx, rY = y0 - 1 + rqy;
        bool ring_on = false;
#pragma unroll
        for (int q = 0; q < NR; ++q)
            if (q == rj) ring_on = on[q];
        return RingItem{rj, rqx, rqy, has_item && rX >= 0 && rX < nx && rY >= 0 && rY < ny && ring_on,
                        xy_mask(rX, rY)};
    };
    const RingItem ring0 = ring_item(0);

    auto phase1 = [&](int zp, bool own) {
        if (zp < 0 || zp >= nz) {
            zero_st(zp);
            return;
        }
        const unsigned zm = z_mask(zp);
        if (own_xy) {
            const unsigned vm = own_mxy & zm;
            T vk[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) vk[k] = ((vm >> k) & 1u) ? T(1) : T(0);
            const T* tvs = tv_slot(zp) + (ty + 1) * TVW + tx + 4;
            T tv[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) tv[k] = tvs[k * SH * TVW];
            if (own) {
                const T* kns = kn_slot(zp) + ty * TX + tx;
                T knw[18];
#pragma unroll
                for (int k = 0; k < 18; ++k) knw[k] = (sc_shell(k) == 0 ? T(2) : T(1)) * kns[k * TY * TX];
                // s_c = sum of n_k and T_c = sum of Tv n_k over existing bonds of shell c
                T sc[2][3], Tc[2][3];
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int a = 0; a < 3; ++a) sc[c][a] = Tc[c][a] = T(0);
#pragma unroll
                for (int k = 0; k < 18; ++k) {
                    const T w = wk<T>(k);
                    const int c = sc_shell(k);
                    const int o[3] = {sc_dx(k), sc_dy(k), sc_dz(k)};
                    const T vt = vk[k] * tv[k];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        if (o[a] == 0) continue;
                        sc[c][a] -= T(o[a]) * w * vk[k];
                        Tc[c][a] -= T(o[a]) * w * vt;
                    }
                }
#pragma unroll
                for (int j = 0; j < NR; ++j)
                    if (on[j]) site_sys(j, tx + 1, ty + 1, zp, vk, tv, knw, std::true_type{}, sc, Tc);
#pragma unroll
                for (int k = 0; k < 18; ++k) tv_next[k] = tv[k];
            } else {
#pragma unroll
                for (int j = 0; j < NR; ++j)
                    if (on[j]) site_sys(j, tx + 1, ty + 1, zp, vk, tv, nullptr, std::false_type{}, nullptr, nullptr);
            }
        }
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const RingItem ri = it == 0 ? ring0 : ring_item(it);
            if (!ri.in) continue;
            const int rj = ri.rj, rqx = ri.rqx, rqy = ri.rqy;
            const unsigned vm = ri.mxy & zm;
            T vk[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) vk[k] = ((vm >> k) & 1u) ? T(1) : T(0);
            const T* tvs = tv_slot(zp) + rqy * TVW + rqx + 3;
            T tv[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) tv[k] = tvs[k * SH * TVW];
            site_sys(rj, rqx, rqy, zp, vk, tv, nullptr, std::false_type{}, nullptr, nullptr);
        }
    };

    // ---------------------------------------------------------------------------------------------- phase 2
    T own_cur[NR][3];
    T tv_cur[18];
    double dot[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) dot[j] = 0.0;

    auto phase2 = [&](int z) {
        if (!own_xy) return;
        const int64_t i = ((int64_t)z * ny + gy) * nx + gx;
        const V2* sm = st_slot(z - 1);
        const V2* s0 = st_slot(z);
        const V2* sp = st_slot(z + 1);
        const int c0 = (ty + 1) * SW + (tx + 1);
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            if (!on[j]) continue;
            const int s = sbase + j;
            T f[3] = {own_cur[j][0], own_cur[j][1], own_cur[j][2]};
#pragma unroll
            for (int k = 0; k < 18; ++k) {
                const V2* pl = sc_dz(k) < 0 ? sm : (sc_dz(k) > 0 ? sp : s0);
                const V2 ba = pl[j * 2 * SPL + sc_shell(k) * SPL + c0 + sc_dy(k) * SW + sc_dx(k)];
                const T gw = tv_cur[k] * ba.x + ba.y;  // zero for bonds that leave the box (see zero_st / init)
                if (sc_dx(k)) f[0] -= T(sc_dx(k)) * gw;
                if (sc_dy(k)) f[1] -= T(sc_dy(k)) * gw;
                if (sc_dz(k)) f[2] -= T(sc_dz(k)) * gw;
            }
            T* o = P.out + ((int64_t)s * P.N + i) * 3;
            if (EPI && P.mask) {
                const uint8_t* mk = P.mask + ((int64_t)(s % P.nmask) * P.N + i) * 3;
                if (!mk[0]) f[0] = T(0);
                if (!mk[1]) f[1] = T(0);
                if (!mk[2]) f[2] = T(0);
            }
            o[0] = f[0];
            o[1] = f[1];
            o[2] = f[2];
            if constexpr (EPI) {
                const T* pu = u_slot(z) + j * UH * UXW + (ty + 2) * UXW + 3 * (tx + 2) + 2;
                dot[j] += (double)pu[0] * (double)f[0] + (double)pu[1] * (double)f[1] + (double)pu[2] * (double)f[2];
            }
        }
    };

    bool ok = true;
    if (any_on) {
        if (tid == 0) {
            for (int p = zbeg - 2; p <= zbeg + 1; ++p) issue_u(p);
            issue_tv(zbeg - 1);
            issue_tv(zbeg);
            issue_kn(zbeg);
            if (zbeg + 1 < zend) issue_kn(zbeg + 1);
        }
        ok = wait_planes(zbeg, zbeg - 1, -1) && wait_planes(zbeg - 1, -1, -1) && wait_planes(zbeg - 2, -1, -1);
        if (ok) {
            phase1(zbeg - 1, false);
            __syncthreads();
            if (tid == 0) {
                fence_proxy_async();
                if (zbeg + 2 <= zend + 1) issue_u(zbeg + 2);
                if (zbeg + 1 <= zend) issue_tv(zbeg + 1);
            }
            ok = wait_planes(zbeg + 1, zbeg, zbeg);
        }
        if (ok) {
            phase1(zbeg, true);
            __syncthreads();
            for (int z = zbeg; z < zend; ++z) {
#pragma unroll
                for (int j = 0; j < NR; ++j)
#pragma unroll
                    for (int a = 0; a < 3; ++a) own_cur[j][a] = own_next[j][a];
#pragma unroll
                for (int k = 0; k < 18; ++k) tv_cur[k] = tv_next[k];
                if (tid == 0) {
                    fence_proxy_async();
                    if (z + 3 <= zend + 1) issue_u(z + 3);
                    if (z + 2 <= zend) issue_tv(z + 2);
                    if (z + 2 < zend) issue_kn(z + 2);
                }
                if (!(ok = wait_planes(z + 2, z + 1, z + 1))) break;
                phase1(z + 1, z + 1 < zend);
                __syncthreads();
                phase2(z);
                __syncthreads();
            }
        }
        if (!ok && tid == 0) {  // let the copies in flight land (bounded) before the block's shared memory is released
            for (int b = 0; b < 8; ++b)
                if ((pend >> b) & 1u) mbar_wait(&bars[b], (ppar >> b) & 1u);
        }
    }

    if constexpr (EPI) {
        if (!P.part) return;
        const int nblk = gridDim.x / P.ngrp;  // CTAs per system
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            if (j >= nr) break;
            const int s = sbase + j;
            const double v = block_sum(ok ? dot[j] : 0.0, red);
            if (tid == 0) {
                P.part[(int64_t)s * nblk + tz] = v;
                __threadfence();
                last_flag = atomicAdd(P.cnt + s, 1u) == (unsigned)(nblk - 1);
            }
            __syncthreads();
            if (last_flag) {
                double acc = 0.0;
                for (int b = tid; b < nblk; b += NTH) acc += __ldcg(P.part + (int64_t)s * nblk + b);
                acc = block_sum(acc, red);
                if (tid == 0) {
                    P.cnt[s] = 0u;
                    if (P.has_sc) cg_alpha_step(P.scv, s, acc, P.it);
                }
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------------------------------ host side
template <typename T>
bool make_map(CUtensorMap* m, const void* base, const uint64_t dims[4], const uint64_t strides_bytes[3],
              const uint32_t box[4])
{
    return make_tensor_map4(m, (int)sizeof(T), base, dims, strides_bytes, box);
}

template <typename T, int NR, int TY, bool EPI>
cudaError_t launch_one(const TmaArgs<T>& a, int ngt, int nzc, cudaStream_t st)
{
    using Lay = Layout<T, NR, TY>;
    const size_t es = sizeof(T);
    const int nset = (a.nsys + a.rhs_per_set - 1) / a.rhs_per_set;
    CUtensorMap mu, mtv, mkn;
    {
        const uint64_t dims[4] = {(uint64_t)3 * a.nx, (uint64_t)a.ny, (uint64_t)a.nz, (uint64_t)a.nsys};
        const uint64_t str[3] = {(uint64_t)3 * a.nx * es, (uint64_t)3 * a.nx * a.ny * es,
                                 (uint64_t)3 * a.nx * a.ny * a.nz * es};
        const uint32_t box[4] = {UXW, (uint32_t)(TY + 4), 1, (uint32_t)NR};
        if (!make_map<T>(&mu, a.u, dims, str, box)) return cudaErrorInvalidValue;
    }
    {
        const uint64_t dims[4] = {(uint64_t)a.nx, (uint64_t)a.ny, (uint64_t)a.nz, (uint64_t)18 * nset};
        const uint64_t str[3] = {(uint64_t)a.nx * es, (uint64_t)a.nx * a.ny * es, (uint64_t)a.nx * a.ny * a.nz * es};
        const uint32_t btv[4] = {TVW, (uint32_t)(TY + 2), 1, 18};
        const uint32_t bkn[4] = {TX, (uint32_t)TY, 1, 18};
        if (!make_map<T>(&mtv, a.Tv, dims, str, btv)) return cudaErrorInvalidValue;
        if (!make_map<T>(&mkn, a.Kn, dims, str, bkn)) return cudaErrorInvalidValue;
    }
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!((attr_set >> dev) & 1ull)) {
        cudaError_t e =
            cudaFuncSetAttribute(k_sc_tma<T, NR, TY, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::BYTES);
        if (e != cudaSuccess) return e;
        attr_set |= 1ull << dev;
    }
    const int ntile = ((a.nx + TX - 1) / TX) * ((a.ny + TY - 1) / TY);
    if (ngt != nset * a.ngrp || (int64_t)a.ngrp * ntile * nzc > 0x7FFFFFFF) return cudaErrorInvalidValue;
    for (int s0 = 0; s0 < nset; s0 += 65535) {
        TmaArgs<T> b = a;
        b.wait_polls = tma_wait_polls();
        b.set0 = s0;
        const int ns = nset - s0 < 65535 ? nset - s0 : 65535;
        k_sc_tma<T, NR, TY, EPI><<<dim3(a.ngrp * ntile * nzc, ns), dim3(TX, TY + RY), Lay::BYTES, st>>>(mu, mtv, mkn,
                                                                                                        b);
    }
    return cudaGetLastError();
}

}  // namespace

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool make_tensor_map4(CUtensorMap* m, int elem_bytes, const void* base, const uint64_t dims[4],
                      const uint64_t strides_bytes[3], const uint32_t box[4])
{
    auto fn = encode_fn();
    if (!fn) return false;
    const uint32_t es[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const CUresult r = fn(m, dt, 4, const_cast<void*>(base), dims, strides_bytes, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool tma_aligned(const void* a, const void* b, const void* c)
{
    return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c)) & 15u) == 0;
}

namespace {
std::atomic<unsigned> g_wait_polls{ptx::kWaitLimit};
}  // namespace

unsigned tma_wait_polls() { return g_wait_polls.load(std::memory_order_relaxed); }
unsigned tma_set_wait_polls(unsigned polls) { return g_wait_polls.exchange(polls); }

bool tma_supported(int nx, int elem_bytes)
{
    // 16-byte global strides for the AoS vectors (3 nx values per row) and the coefficient planes (nx per row)
    if (elem_bytes == 4 && nx % 4 != 0) return false;
    if (elem_bytes == 8 && nx % 2 != 0) return false;
    return encode_fn() != nullptr;
}

int tma_group_size(int rhs_per_set, int elem_bytes)
{
    // FP64: two systems per CTA (198 KB of shared memory; three do not fit), so a set's coefficients cross HBM half
    // as often
    if (elem_bytes == 8) return rhs_per_set >= 2 ? 2 : 1;
    for (int g = 3; g > 1; --g)
        if (rhs_per_set % g == 0) return g;
    return rhs_per_set >= 3 ? 3 : rhs_per_set;
}

int tma_tile_rows(int elem_bytes) { return elem_bytes == 8 ? 4 : 8; }

int tma_zchunk(int nx, int ny, int nz, int nset, int ngrp, int elem_bytes)
{
    const int ty = tma_tile_rows(elem_bytes);
    const long long base = (long long)((nx + TX - 1) / TX) * ((ny + ty - 1) / ty) * nset * ngrp;
    int nzc = 1;
    while (base * nzc < 2 * 148 && nz / (nzc + 1) >= 8) ++nzc;
    return (nz + nzc - 1) / nzc;
}

int tma_dot_blocks_max(int nx, int ny, int nz, int elem_bytes)
{
    const int ty = tma_tile_rows(elem_bytes);
    return ((nx + TX - 1) / TX) * ((ny + ty - 1) / ty) * (nz / 8 + 1);
}

template <typename T>
cudaError_t launch_sc_tma(const TmaArgs<T>& a, bool epi, cudaStream_t st)
{
    const int nset = (a.nsys + a.rhs_per_set - 1) / a.rhs_per_set;
    const int ngt = nset * a.ngrp;
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    if constexpr (sizeof(T) == 8) {
        switch (a.nr) {
        case 1: return epi ? launch_one<T, 1, 4, true>(a, ngt, nzc, st) : launch_one<T, 1, 4, false>(a, ngt, nzc, st);
        case 2: return epi ? launch_one<T, 2, 4, true>(a, ngt, nzc, st) : launch_one<T, 2, 4, false>(a, ngt, nzc, st);
        default: return cudaErrorInvalidValue;
        }
    } else {
        switch (a.nr) {
        case 1: return epi ? launch_one<T, 1, 8, true>(a, ngt, nzc, st) : launch_one<T, 1, 8, false>(a, ngt, nzc, st);
        case 2: return epi ? launch_one<T, 2, 8, true>(a, ngt, nzc, st) : launch_one<T, 2, 8, false>(a, ngt, nzc, st);
        case 3: return epi ? launch_one<T, 3, 8, true>(a, ngt, nzc, st) : launch_one<T, 3, 8, false>(a, ngt, nzc, st);
        default: return cudaErrorInvalidValue;
        }
    }
}

template cudaError_t launch_sc_tma<float>(const TmaArgs<float>&, bool, cudaStream_t);
template cudaError_t launch_sc_tma<double>(const TmaArgs<double>&, bool, cudaStream_t);

}  // namespace lpm
