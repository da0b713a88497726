// Pair-packed TMA-fed SC operator for the FP32 CG engine: out = K u for the two systems of a pair at once.
//
// Same decomposition as the TMA operator (code-force form of coarse3d/lin3d.py:126-149):
//   f_i   = own_i + sum_k n_k (A_q^c + Tv_ik B_q^c),   A = TS/2, B = S/2 (shell-1 values pre-scaled by 1/sqrt2)
//   own_i = sum_k 2 Kn_ik dL_ik n_k + sum_c (A_i^c s_i^c + B_i^c T_i^c)
// but the two systems of a pair travel together in one 64-bit register and are processed by the packed FP32x2
// instructions of sm_100a (add/sub/mul/fma .rn.f32x2): every shared-memory load of u and every add or FMA on a
// displacement-dependent quantity serves both systems, and the bond coefficients (shared by the pair) are loaded
// once.
//
// Vector layout ("pair layout"): (npair, N, 3, 2) FP32, element (pair, i, a, lane), pair = set * npp + j / 2 and
// lane = j % 2 for system j of a coefficient set (npp = ceil(rhs_per_set / 2)).  The second lane of the last pair of
// a set with an odd number of systems is a dummy the caller keeps at zero.
//
// The output is not masked: the CG engine keeps p zero on fixed DOFs (so p.Ap needs no mask) and masks Ap where it
// updates r.
//
// Tile: 16 x 16 sites, 256 threads; a warp covers rows ty and ty + 2 of 16 columns (the two half-warps then read
// Tv rows 48 floats apart: no shared-memory bank conflicts).  The CTA marches in z over a chunk of planes; step z
// computes the shell sums of plane z+1 (tile + 1-site ring) with the own terms of the tile (phase 1), then the
// neighbour terms and the output of plane z (phase 2).  Shared memory of the staged variant, 207 KB (one CTA per SM):
//   u      : 5 planes x 20 rows x 120 floats (sites x0-2 .. x0+17, pair layout)
//   Tv     : 2 planes x 18 slots x 18 rows x 24 sites (x0-4 .. x0+19)
//   Kn     : 2 planes x 18 slots x 16 rows x 24 sites (x0 .. x0+23)
//   (B, A) : 4 planes x 2 shells x 18 x 18 sites x float4 {B lane 0, B lane 1, A lane 0, A lane 1}
// All global inputs arrive by TMA (no multicast), issued by one thread a plane ahead into rings guarded by
// mbarriers.  Bonds that leave the box: in warps where every lane's site has all 18 bonds no masking is done;
// otherwise dL of missing bonds is zeroed by selection, so whatever the coefficients of missing bonds hold is
// multiplied by zero, as in the reference.  (B, A) of sites outside the box is zero.  Every mbarrier wait is bounded;
// on expiry the kernel records an error code, waits (bounded) for the copies it issued, and stops computing.
//
// Epilogues (PairMode): PM_NONE writes f = K u; PM_DOT also forms per-system u.f partials in FP32 per thread, reduced
// in FP64 deterministically, and the last block of a system runs the CG alpha step.  The smoother epilogues of the
// AMG preconditioner take a right-hand side b (pair layout) and each lane's free box: PM_RESID writes the masked
// residual m (b - K u), PM_SMOOTH the damped block-Jacobi sweep u + w m M (b - K u) with the 3x3 inverse M of the
// site (u from the shared-memory tile), and PM_SMOOTH_DOT adds b.out per system and the PCG beta step.
#include <cudaTypedefs.h>

#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "lpm_fused.h"
#include "lpm_ptx.cuh"
#include "lpm_tma.h"

namespace lpm {

namespace {

using namespace ptx;

constexpr int PX = 16, PY = 16, PNT = PX * PY;
constexpr int PUW = 6 * (PX + 4);  // floats per u row: sites x0-2 .. x0+17, 3 components x 2 lanes
constexpr int PUWE = 3 * (PX + 4); // u elements (8-byte lane groups: an FP32 pair or one FP64 value) per row
constexpr int PUH = PY + 4;        // u rows y0-2 .. y0+17
constexpr int PSW = PX + 2, PSH = PY + 2, PSPL = PSW * PSH;  // tile + 1-site ring
constexpr int PTVW = 24;           // Tv sites per row (x0-4 .. x0+19)
constexpr int PKNW = 24;           // Kn sites per row (x0 .. x0+23)
constexpr int PNRING = PSPL - PNT;
// Threads per CTA.  Lean: the 256 tile threads also take the 68 ring sites (threads 0..67).  Staged: three more warps
// own the ring sites (threads 256..323), so the tile warps carry no ring work and phase 1 costs every warp about the
// same; an idle lane of the last ring warp issues the TMA fills, off the tile warps' path.
#ifndef LPM_PAIR_RING_THREADS
#define LPM_PAIR_RING_THREADS 96
#endif
constexpr int PRING_THREADS = LPM_PAIR_RING_THREADS;  // ring threads of the staged variant (a multiple of 32)
constexpr int PRING_ITEMS = (PNRING + PRING_THREADS - 1) / PRING_THREADS;  // ring sites per ring thread (at most)
__host__ __device__ constexpr int pair_threads(bool lean) { return lean ? PNT : PNT + PRING_THREADS; }
static_assert(PRING_THREADS % 32 == 0 && PRING_THREADS >= 32, "whole ring warps");
constexpr unsigned FULL18 = 0x3FFFFu;

constexpr size_t PU_SLOT = (size_t)PUH * PUW * 4;
constexpr size_t PTV_SLOT = (size_t)18 * PSH * PTVW * 4;  // FP32 coefficients; FP64 doubles it (tv_slot_bytes)
constexpr size_t PKN_SLOT = (size_t)18 * PY * PKNW * 4;
constexpr size_t PBA_SLOT = (size_t)2 * PSPL * 16;
// Two variants share the kernel.  Staged (LEAN = false): Tv double-buffered and Kn staged by TMA, five u planes and
// four (B, A) planes, so that one block barrier per z step suffices (a warp may start the next step's phase 1 while
// others finish phase 2), 207 KB, one CTA per SM.  Lean (LEAN = true): one Tv slot refilled right after phase 1 has
// read it, Kn of the own sites read from global memory in phase 1 and Tv of the own sites from global memory (L2) in
// phase 2, four u and three (B, A) planes with two block barriers per step, 101 KB and at most 128 registers: two
// CTAs (16 warps) per SM.
//
// FP64 (CT = double): the same kernel for one FP64 system per lane group ("pair" = one system), on natural-layout
// vectors (nsys, N, 3), which are this layout with one lane.  Only the lean variant: the staged rings of doubled
// coefficient planes would not fit (131 KB lean, one CTA per SM).
__host__ __device__ constexpr int u_slots(bool lean) { return lean ? 4 : 5; }
__host__ __device__ constexpr int ba_slots(bool lean) { return lean ? 3 : 4; }
__host__ __device__ constexpr int tv_slots(bool lean) { return lean ? 1 : 2; }
__host__ __device__ constexpr size_t tv_slot_bytes(int es) { return PTV_SLOT / 4 * es; }
__host__ __device__ constexpr size_t kn_slot_bytes(int es) { return PKN_SLOT / 4 * es; }
__host__ __device__ constexpr size_t off_tv(bool lean) { return u_slots(lean) * PU_SLOT; }
__host__ __device__ constexpr size_t off_kn(bool lean, int es = 4)
{
    return off_tv(lean) + tv_slots(lean) * tv_slot_bytes(es);
}
__host__ __device__ constexpr size_t off_ba(bool lean, int es = 4)
{
    return off_kn(lean, es) + (lean ? 0 : 2 * kn_slot_bytes(es));
}
__host__ __device__ constexpr size_t pair_bytes(bool lean, int es = 4)
{
    return off_ba(lean, es) + ba_slots(lean) * PBA_SLOT;
}
static_assert(PU_SLOT % 128 == 0 && PTV_SLOT % 128 == 0 && PKN_SLOT % 128 == 0 && PBA_SLOT % 128 == 0,
              "TMA destinations must stay 128-byte aligned");
static_assert(pair_bytes(false) <= 227 * 1024, "shared memory budget");
static_assert(2 * (pair_bytes(true) + 2048) <= 228 * 1024, "two lean CTAs per SM");
static_assert(pair_bytes(true, 8) <= 227 * 1024, "FP64 lean shared memory budget");

// Lane type of a coefficient type: FP32 -> a packed pair of two systems, FP64 -> one system.
template <typename CT>
struct PairLane;
template <>
struct PairLane<float> {
    using V = pair_t;
    using BA = float4;  // {B lane 0, B lane 1, A lane 0, A lane 1}
    static constexpr int NL = 2;
    static __device__ __forceinline__ BA make_ba(V b, V a)
    {
        float bl, bh, al, ah;
        unpk(b, bl, bh);
        unpk(a, al, ah);
        return make_float4(bl, bh, al, ah);
    }
    static __device__ __forceinline__ V b_of(const BA& v) { return pk(v.x, v.y); }
    static __device__ __forceinline__ V a_of(const BA& v) { return pk(v.z, v.w); }
    static __device__ __forceinline__ BA zero_ba() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    static __device__ __forceinline__ void lanes(V v, float& l0, float& l1) { unpk(v, l0, l1); }
};
template <>
struct PairLane<double> {
    using V = double;
    using BA = double2;  // {B, A}
    static constexpr int NL = 1;
    static __device__ __forceinline__ BA make_ba(V b, V a) { return make_double2(b, a); }
    static __device__ __forceinline__ V b_of(const BA& v) { return v.x; }
    static __device__ __forceinline__ V a_of(const BA& v) { return v.y; }
    static __device__ __forceinline__ BA zero_ba() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ void lanes(V v, double& l0, double& l1)
    {
        l0 = v;
        l1 = 0.0;
    }
};

__host__ __device__ constexpr unsigned dir_bits(int axis, int sgn)
{
    unsigned m = 0;
    for (int k = 0; k < 18; ++k) {
        const int d = axis == 0 ? sc_dx(k) : axis == 1 ? sc_dy(k) : sc_dz(k);
        if (d == sgn) m |= 1u << k;
    }
    return m;
}

// Slot geometry: for axis slots (shell 0) the component a and sign sa; for diagonal slots (shell 1) the two
// components a < b, their signs and the plane index of the pair (0: xy, 1: xz, 2: yz).
struct SlotGeo {
    int a, b, sa, sb, plane;
};
__host__ __device__ constexpr SlotGeo slot_geo(int k)
{
    const int o[3] = {sc_dx(k), sc_dy(k), sc_dz(k)};
    SlotGeo g{-1, -1, 0, 0, -1};
    for (int c = 0; c < 3; ++c) {
        if (o[c] == 0) continue;
        if (g.a < 0) {
            g.a = c;
            g.sa = o[c];
        } else {
            g.b = c;
            g.sb = o[c];
        }
    }
    if (g.b >= 0) g.plane = g.a == 0 ? (g.b == 1 ? 0 : 1) : 2;
    return g;
}


template <int MODE, bool LEAN, typename CT = float>
__global__ void __launch_bounds__(pair_threads(LEAN), (LEAN && sizeof(CT) == 4) ? 2 : 1)
    k_sc_pair(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_tv,
              const __grid_constant__ CUtensorMap tm_kn, PairArgs P)
{
    static_assert(sizeof(CT) == 4 || (LEAN && MODE <= PM_DOT), "FP64: lean variant, plain and dot epilogues only");
    using LN = PairLane<CT>;
    using V = typename LN::V;
    using BA = typename LN::BA;
    constexpr int NL = LN::NL;
    constexpr int ES = (int)sizeof(CT);
    constexpr V VZ = V(0);
    // FP64 lean: the own site's Tv of phase 2 (read from global memory, L2) is loaded before the block barrier that
    // ends phase 1, so the loads are in flight while the block waits; the FP32 lean variant has no registers to spare.
    constexpr bool PREF_TV = LEAN && sizeof(CT) == 8;
    // Likewise its Kn of phase 1 is loaded at the top of the step, before the waits for the step's fills.
    constexpr bool PREF_KN = LEAN && sizeof(CT) == 8;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int NUS = u_slots(LEAN), NBAS = ba_slots(LEAN);
    constexpr int BTV = NUS, BKN = NUS + 2, NBAR = NUS + 4;  // mbarriers: u 0..NUS-1, Tv BTV.., Kn BKN..
    __shared__ __align__(8) uint64_t bars[NBAR];
    __shared__ double red[32];
    __shared__ int abort_flag;  // set before the first block barrier only (shared-memory alignment check)
    __shared__ bool last_flag;

    V* su = reinterpret_cast<V*>(smem);  // u elements: (slot, PUH rows, PUWE)
    CT* stv = reinterpret_cast<CT*>(smem + off_tv(LEAN));
    CT* skn = reinterpret_cast<CT*>(smem + off_kn(LEAN, ES));
    BA* sba = reinterpret_cast<BA*>(smem + off_ba(LEAN, ES));
    constexpr size_t TVS = tv_slot_bytes(ES) / ES, KNS = kn_slot_bytes(ES) / ES;  // elements per Tv / Kn slot
    constexpr size_t US = PU_SLOT / 8, BAS = PBA_SLOT / 16;                     // elements per u / (B, A) slot

    constexpr int NTH = pair_threads(LEAN);
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const bool tile_thr = tid < PNT;  // owns a site of the tile (all threads of the lean variant)
    const int tx = lane & 15, ty = ((wid >> 1) << 2) + (wid & 1) + ((lane >> 4) << 1);
    // the thread that issues the TMA fills and tracks them for the drain on abort
    const bool producer = tid == (LEAN ? 0 : NTH - 1);
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int ntx = (nx + PX - 1) / PX, nty = (ny + PY - 1) / PY;
    // Grid: x = (pair of the set, column tile, z chunk) with the pair fastest, y = coefficient set.  The pairs of a set
    // are adjacent in launch order, so they run together and the second and later pairs find the set's coefficient
    // tiles in L2 (with the pairs far apart, a batch too large for L2 streams the coefficients once per pair).
    const int jp = blockIdx.x % P.npp, tz = blockIdx.x / P.npp;  // tz: this CTA's block index within its system
    const int tile = tz % (ntx * nty), zc = tz / (ntx * nty);
    const int x0 = (tile % ntx) * PX, y0 = (tile / ntx) * PY;
    const int set = blockIdx.y + P.set0;
    const int pr = set * P.npp + jp;
    const int sbase = set * P.rhs_per_set + NL * jp;
    int nr = P.rhs_per_set - NL * jp;
    nr = nr < NL ? nr : NL;
    if (sbase + nr > P.nsys) nr = P.nsys - sbase;
    const int zbeg = zc * P.zchunk;
    const int zend = min(nz, zbeg + P.zchunk);
    const bool on0 = nr > 0 && (!P.act || P.act[sbase]);
    const bool on1 = nr > 1 && (!P.act || P.act[sbase + 1]);
    bool any_on = on0 || on1;
    constexpr bool EPI = MODE == PM_DOT || MODE == PM_SMOOTH_DOT;
    constexpr bool SMOOTH = MODE == PM_SMOOTH || MODE == PM_SMOOTH_DOT;
    // free boxes and weights of the two lanes (smoother epilogues); a dummy lane has an empty box
    int bl0[3] = {0, 0, 0}, bh0[3] = {-1, -1, -1}, bl1[3] = {0, 0, 0}, bh1[3] = {-1, -1, -1};
    float w0 = 0.f, w1 = 0.f;
    if constexpr (MODE >= PM_RESID) {
        if (nr > 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                bl0[a] = P.fbox[6 * sbase + a];
                bh0[a] = P.fbox[6 * sbase + 3 + a];
            }
            if (SMOOTH) w0 = P.fw[sbase];
        }
        if (nr > 1) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                bl1[a] = P.fbox[6 * sbase + 6 + a];
                bh1[a] = P.fbox[6 * sbase + 9 + a];
            }
            if (SMOOTH) w1 = P.fw[sbase + 1];
        }
    }

    if (tid == 0) {
        for (int b = 0; b < NBAR; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
        abort_flag = 0;
        if (saddr(smem) & 127u) {  // TMA destinations must be 128-byte aligned: refuse to run and report
            abort_flag = 1;
            if (P.err) atomicExch(P.err, 2);
        }
    }
    {
        for (int e = tid; e < NBAS * 2 * PSPL; e += NTH) sba[e] = LN::zero_ba();
        // u slots standing for planes below 0 are never loaded; keep them finite
        const int nneg = zbeg - 2 < 0 ? 2 - zbeg : 0;
        for (int e = tid; e < nneg * (int)US; e += NTH) su[e] = VZ;
    }
    __syncthreads();
    if (abort_flag) any_on = false;

    // ------------------------------------------------------------------------------------------ producer side
    // Fill n of a stream lands in slot n % nslots with mbarrier parity (n / nslots) & 1.  Thread 0 issues and keeps
    // the outstanding fills of each barrier in `pend` (bit b) / `ppar` (parity), for the drain on abort.
    const int u0 = zbeg - 2, tv0 = zbeg - 1, kn0 = zbeg;
    unsigned pend = 0, ppar = 0;
    auto note = [&](int b, int parity) {
        pend |= 1u << b;
        ppar = (ppar & ~(1u << b)) | ((unsigned)parity << b);
    };
    auto issue_u = [&](int p) {
        const int n = p - u0;
        uint64_t* bar = &bars[n % NUS];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, (uint32_t)PU_SLOT);
        tma_load4(su + (size_t)(n % NUS) * US, &tm_u, bar, 3 * NL * (x0 - 2), y0 - 2, p, pr);
        note(n % NUS, (n / NUS) & 1);
    };
    // Tv fill n: slot n % tv_slots, barrier BTV + slot, parity (n / tv_slots) & 1
    constexpr int NTV = tv_slots(LEAN);
    auto issue_tv = [&](int p) {
        const int n = p - tv0;
        uint64_t* bar = &bars[BTV + n % NTV];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, (uint32_t)tv_slot_bytes(ES));
        tma_load4(stv + (size_t)(n % NTV) * TVS, &tm_tv, bar, x0 - 4, y0 - 1, p, 18 * set);
        note(BTV + n % NTV, (n / NTV) & 1);
    };
    auto issue_kn = [&](int p) {
        const int n = p - kn0;
        uint64_t* bar = &bars[BKN + (n & 1)];
        if (p < 0 || p >= nz) {
            mbar_arrive(bar);
            return;
        }
        mbar_expect_arrive(bar, (uint32_t)kn_slot_bytes(ES));
        tma_load4(skn + (size_t)(n & 1) * KNS, &tm_kn, bar, x0, y0, p, 18 * set);
        note(BKN + (n & 1), (n >> 1) & 1);
    };
    // Every thread waits (bounded) for the in-range fills it is about to read; an expired wait sets the thread's own
    // `lost` flag, and the next block barrier ORs the flags of all threads (__syncthreads_or), so every thread takes
    // the same abort decision at the same barrier.  A shared flag would not do: a fast warp could raise it for step
    // z+1 before a slow warp has read it after step z's barrier, and the two would then wait at different barriers.
    bool lost = false;
    auto wait_fill = [&](int b, int parity) {
        if (!mbar_wait(&bars[b], (uint32_t)parity, P.wait_polls)) {
            lost = true;
            if (P.err) atomicExch(P.err, 1);
        } else if (producer) {
            pend &= ~(1u << b);
        }
    };
    auto wait_planes = [&](int pu, int ptv, int pkn) {
        if (pu >= 0 && pu < nz && pu >= u0) wait_fill((pu - u0) % NUS, ((pu - u0) / NUS) & 1);
        if (ptv >= 0 && ptv < nz && ptv >= tv0) wait_fill(BTV + (ptv - tv0) % NTV, ((ptv - tv0) / NTV) & 1);
        if (!LEAN && pkn >= 0 && pkn < nz && pkn >= kn0 && pkn < zend)
            wait_fill(BKN + ((pkn - kn0) & 1), ((pkn - kn0) >> 1) & 1);
    };

    auto u_slot = [&](int p) { return su + (size_t)((p - u0) % NUS) * US; };
    auto tv_slot = [&](int p) { return stv + (size_t)((p - tv0) % NTV) * TVS; };
    auto kn_slot = [&](int p) { return skn + (size_t)((p - kn0) & 1) * KNS; };
    auto ba_slot = [&](int p) { return sba + (size_t)(((p % NBAS) + NBAS) % NBAS) * BAS; };

    // ---------------------------------------------------------------------------------------------- phase 1
    // Shell sums of the site (qx, qy) (ring coordinates, 0 = x0-1 / y0-1) of plane zp for both lanes, stored as
    // (B, A); with OWN also the own terms.  Slot loop fully unrolled; signs are compile-time, so every accumulation is
    // an add or FMA into a "plus" or "minus" accumulator.  Diagonal slots use d' = o.(u_q - u_i) unscaled.
    V own_next[3] = {VZ, VZ, VZ};
    CT tv_next[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) tv_next[k] = CT(0);
    CT kn_pre[18];  // PREF_KN: the own site's Kn of the next phase 1

    // pm, p0, pp: the u slots of planes zp-1, zp, zp+1; bsl: the (B, A) slot of plane zp.
    auto site = [&](auto own_tag, auto mask_tag, int qx, int qy, const V* pm, const V* p0, const V* pp, BA* bsl,
                    unsigned vm, const CT* tvs, const CT* kns, int64_t kst) {
        constexpr bool OWN = decltype(own_tag)::value;
        constexpr bool MASKED = decltype(mask_tag)::value;
        const int ci = (qy + 1) * PUWE + 3 * (qx + 1);
        const V ui[3] = {p0[ci], p0[ci + 1], p0[ci + 2]};
        const V cpl[3] = {add2(ui[0], ui[1]), add2(ui[0], ui[2]), add2(ui[1], ui[2])};
        const V cmi[3] = {sub2(ui[0], ui[1]), sub2(ui[0], ui[2]), sub2(ui[1], ui[2])};
        V Sp0 = VZ, Sm0 = VZ, Sp1 = VZ, Sm1 = VZ, Tp0 = VZ, Tm0 = VZ, Tp1 = VZ, Tm1 = VZ;
        V fp[3] = {VZ, VZ, VZ}, fm[3] = {VZ, VZ, VZ};
        CT s0[3] = {0, 0, 0}, s1[3] = {0, 0, 0}, T0[3] = {0, 0, 0}, T1[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < 18; ++k) {
            const SlotGeo g = slot_geo(k);
            const V* pl = sc_dz(k) < 0 ? pm : (sc_dz(k) > 0 ? pp : p0);
            const int qo = ci + sc_dy(k) * PUWE + 3 * sc_dx(k);
            const CT tv = tvs[k * PSH * PTVW];
            const bool vb = !MASKED || ((vm >> k) & 1u);
            if (sc_shell(k) == 0) {
                V t = sub2(pl[qo + g.a], ui[g.a]);  // u_q,a - u_i,a ; dL = sa t
                if (MASKED && !vb) t = VZ;
                if (g.sa > 0) {
                    Sp0 = add2(Sp0, t);
                    Tp0 = fma2(dup(tv), t, Tp0);
                } else {
                    Sm0 = add2(Sm0, t);
                    Tm0 = fma2(dup(tv), t, Tm0);
                }
                if constexpr (OWN) {
                    const CT kn = PREF_KN ? kn_pre[k] : (LEAN ? __ldg(kns + k * kst) : kns[k * kst]);
                    fm[g.a] = fma2(dup(CT(2) * kn), t, fm[g.a]);  // f_a -= 2 Kn t
                    if (vb) {
                        s0[g.a] -= (CT)g.sa;
                        T0[g.a] -= (CT)g.sa * tv;
                    }
                }
            } else {
                const V qa = pl[qo + g.a], qb = pl[qo + g.b];
                // d' = sa t with t = (u_q,a +- u_q,b) - (u_i,a +- u_i,b)
                V t = g.sa == g.sb ? sub2(add2(qa, qb), cpl[g.plane]) : sub2(sub2(qa, qb), cmi[g.plane]);
                if (MASKED && !vb) t = VZ;
                if (g.sa > 0) {
                    Sp1 = add2(Sp1, t);
                    Tp1 = fma2(dup(tv), t, Tp1);
                } else {
                    Sm1 = add2(Sm1, t);
                    Tm1 = fma2(dup(tv), t, Tm1);
                }
                if constexpr (OWN) {
                    const CT kn = PREF_KN ? kn_pre[k] : (LEAN ? __ldg(kns + k * kst) : kns[k * kst]);
                    const V kn2 = dup(kn);
                    fm[g.a] = fma2(kn2, t, fm[g.a]);  // f_a -= sa Kn d' = Kn t
                    if (g.sa == g.sb)
                        fm[g.b] = fma2(kn2, t, fm[g.b]);
                    else
                        fp[g.b] = fma2(kn2, t, fp[g.b]);
                    if (vb) {
                        s1[g.a] -= (CT)g.sa;
                        s1[g.b] -= (CT)g.sb;
                        T1[g.a] -= (CT)g.sa * tv;
                        T1[g.b] -= (CT)g.sb * tv;
                    }
                }
            }
            if constexpr (OWN && !LEAN) tv_next[k] = tv;
        }
        // B0 = S0/2, A0 = TS0/2; shell 1 pre-scaled by 1/sqrt2: B1w = S1'/4, A1w = TS1'/4
        const V h = dup(CT(0.5)), q = dup(CT(0.25));
        const V B0 = mul2(h, sub2(Sp0, Sm0)), A0 = mul2(h, sub2(Tp0, Tm0));
        const V B1 = mul2(q, sub2(Sp1, Sm1)), A1 = mul2(q, sub2(Tp1, Tm1));
        BA* dst = bsl + qy * PSW + qx;
        dst[0] = LN::make_ba(B0, A0);
        dst[PSPL] = LN::make_ba(B1, A1);
        if constexpr (OWN) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                V o = sub2(fp[a], fm[a]);
                o = fma2(B0, dup(T0[a]), o);
                o = fma2(B1, dup(T1[a]), o);
                if constexpr (MASKED) {  // s_c vanishes for a site with all bonds
                    o = fma2(A0, dup(s0[a]), o);
                    o = fma2(A1, dup(s1[a]), o);
                }
                own_next[a] = o;
            }
        }
    };

    constexpr unsigned XN = dir_bits(0, -1), XP = dir_bits(0, 1), YN = dir_bits(1, -1), YP = dir_bits(1, 1),
                       ZN = dir_bits(2, -1), ZP = dir_bits(2, 1);
    auto xy_mask = [&](int X, int Y) {
        unsigned m = FULL18;
        if (X == 0) m &= ~XN;
        if (X == nx - 1) m &= ~XP;
        if (Y == 0) m &= ~YN;
        if (Y == ny - 1) m &= ~YP;
        return m;
    };
    auto z_mask = [&](int z) {
        unsigned m = FULL18;
        if (z == 0) m &= ~ZN;
        if (z == nz - 1) m &= ~ZP;
        return m;
    };

    const int gx = x0 + tx, gy = y0 + ty;
    const bool own_xy = tile_thr && gx < nx && gy < ny;
    const unsigned own_mxy = xy_mask(gx, gy);
    // Ring sites of this thread: items rit, rit + RSTR, ... (lean: the tile threads 0..67 take one each; staged: the
    // ring threads take PRING_ITEMS at most).  Item geometry: position in the ring, inside the box, box-edge mask.
    const int rit = LEAN ? tid : tid - PNT;
    constexpr int RSTR = LEAN ? PNT : PRING_THREADS;
    constexpr int RITEMS = LEAN ? 1 : PRING_ITEMS;
    struct RingSite {
        int qx, qy;
        bool in;
        unsigned mxy;
    };
    auto ring_site = [&](int it) {
        RingSite r{0, 0, false, 0u};
        if (it < 0 || it >= PNRING) return r;
        if (it < PSW) {
            r.qx = it;
            r.qy = 0;
        } else if (it < 2 * PSW) {
            r.qx = it - PSW;
            r.qy = PSH - 1;
        } else if (it < 2 * PSW + PY) {
            r.qx = 0;
            r.qy = it - 2 * PSW + 1;
        } else {
            r.qx = PSW - 1;
            r.qy = it - 2 * PSW - PY + 1;
        }
        const int X = x0 - 1 + r.qx, Y = y0 - 1 + r.qy;
        r.in = X >= 0 && X < nx && Y >= 0 && Y < ny;
        r.mxy = xy_mask(X, Y);
        return r;
    };
    RingSite rs[RITEMS];
#pragma unroll
    for (int j = 0; j < RITEMS; ++j) rs[j] = ring_site(rit >= 0 ? rit + j * RSTR : -1);  // tile threads: none

    using T_ = std::true_type;
    using F_ = std::false_type;
    auto load_kn = [&](int zp) {  // PREF_KN: the own site's Kn of plane zp into kn_pre
        if constexpr (PREF_KN) {
            if (own_xy && zp >= 0 && zp < nz) {
                const CT* kg = reinterpret_cast<const CT*>(P.Kn) + (int64_t)18 * set * P.N +
                               ((int64_t)zp * ny + gy) * nx + gx;
#pragma unroll
                for (int k = 0; k < 18; ++k) kn_pre[k] = __ldg(kg + (int64_t)k * P.N);
            }
        }
    };
    // Phase 1 of plane zp: pm, p0, pp are its u slots (planes zp-1, zp, zp+1), tvsl / knsl its Tv / Kn slots and bsl
    // its (B, A) slot.
    auto phase1 = [&](int zp, bool own, const V* pm, const V* p0, const V* pp, const CT* tvsl, const CT* knsl,
                      BA* bsl) {
        if (zp < 0 || zp >= nz) {
            for (int e = tid; e < 2 * PSPL; e += NTH) bsl[e] = LN::zero_ba();
            return;
        }
        const unsigned zm = z_mask(zp);
        const unsigned vm = own_mxy & zm;
        const bool uni = __all_sync(0xffffffffu, !own_xy || vm == FULL18);
        if (own_xy) {
            const CT* tvs = tvsl + (ty + 1) * PTVW + tx + 4;
            if (own) {
                const CT* kns;
                int64_t kst;
                if constexpr (LEAN) {
                    kns = reinterpret_cast<const CT*>(P.Kn) + (int64_t)18 * set * P.N + ((int64_t)zp * ny + gy) * nx +
                          gx;
                    kst = P.N;
                } else {
                    kns = knsl + ty * PKNW + tx;
                    kst = PY * PKNW;
                }
                if (uni)
                    site(T_{}, F_{}, tx + 1, ty + 1, pm, p0, pp, bsl, vm, tvs, kns, kst);
                else
                    site(T_{}, T_{}, tx + 1, ty + 1, pm, p0, pp, bsl, vm, tvs, kns, kst);
            } else {
                if (uni)
                    site(F_{}, F_{}, tx + 1, ty + 1, pm, p0, pp, bsl, vm, tvs, nullptr, 0);
                else
                    site(F_{}, T_{}, tx + 1, ty + 1, pm, p0, pp, bsl, vm, tvs, nullptr, 0);
            }
        }
#pragma unroll
        for (int j = 0; j < RITEMS; ++j) {
        const int rqx = rs[j].qx, rqy = rs[j].qy;
        const bool ring_in = rs[j].in;
        const unsigned rvm = rs[j].mxy & zm;
        const bool runi = __all_sync(0xffffffffu, !ring_in || rvm == FULL18);
        if (ring_in) {
            const CT* tvs = tvsl + rqy * PTVW + rqx + 3;
            if (runi)
                site(F_{}, F_{}, rqx, rqy, pm, p0, pp, bsl, rvm, tvs, nullptr, 0);
            else
                site(F_{}, T_{}, rqx, rqy, pm, p0, pp, bsl, rvm, tvs, nullptr, 0);
        }
        }
    };

    // ---------------------------------------------------------------------------------------------- phase 2
    V own_cur[3] = {VZ, VZ, VZ};
    CT tv_cur[18];
    V dotp = VZ;
    // Phase 2 of plane z: bm, b0, bp are the (B, A) slots of planes z-1, z, z+1 and uz the u slot of plane z.
    auto phase2 = [&](int z, const BA* bm, const BA* b0, const BA* bp, const V* uz) {
        if (!own_xy) return;
        const int64_t i = ((int64_t)z * ny + gy) * nx + gx;
        const int c0 = (ty + 1) * PSW + (tx + 1);
        V f[3] = {own_cur[0], own_cur[1], own_cur[2]};
        const CT* tvg = reinterpret_cast<const CT*>(P.Tv) + (int64_t)18 * set * P.N + i;
#pragma unroll
        for (int k = 0; k < 18; ++k) {
            const SlotGeo g = slot_geo(k);
            const BA* pl = sc_dz(k) < 0 ? bm : (sc_dz(k) > 0 ? bp : b0);
            const BA v = pl[sc_shell(k) * PSPL + c0 + sc_dy(k) * PSW + sc_dx(k)];
            const CT tvk = (LEAN && !PREF_TV) ? __ldg(tvg + (int64_t)k * P.N) : tv_cur[k];
            const V gw = fma2(dup(tvk), LN::b_of(v), LN::a_of(v));  // zero for bonds leaving the box
            f[g.a] = g.sa > 0 ? sub2(f[g.a], gw) : add2(f[g.a], gw);
            if (sc_shell(k) == 1) f[g.b] = g.sb > 0 ? sub2(f[g.b], gw) : add2(f[g.b], gw);
        }
        V* o = reinterpret_cast<V*>(P.out) + ((int64_t)pr * P.N + i) * 3;
        if constexpr (MODE <= PM_DOT) {
            o[0] = f[0];
            o[1] = f[1];
            o[2] = f[2];
            if constexpr (EPI) {
                const V* pu = uz + (ty + 2) * PUWE + 3 * (tx + 2);
                dotp = fma2(pu[0], f[0], dotp);
                dotp = fma2(pu[1], f[1], dotp);
                dotp = fma2(pu[2], f[2], dotp);
            }
        } else if constexpr (NL == 2) {
            const bool in0 = gx >= bl0[0] && gx <= bh0[0] && gy >= bl0[1] && gy <= bh0[1] && z >= bl0[2] &&
                             z <= bh0[2];
            const bool in1 = gx >= bl1[0] && gx <= bh1[0] && gy >= bl1[1] && gy <= bh1[1] && z >= bl1[2] &&
                             z <= bh1[2];
            const pair_t* rh = reinterpret_cast<const pair_t*>(P.rhs + (((int64_t)pr * P.N + i) * 3) * 2);
            float t0[3], t1[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) unpk(sub2(rh[a], f[a]), t0[a], t1[a]);
            if constexpr (MODE == PM_RESID) {
#pragma unroll
                for (int a = 0; a < 3; ++a) o[a] = pk(in0 ? t0[a] : 0.f, in1 ? t1[a] : 0.f);
            } else {
                const float* ms = P.Ms + (int64_t)set * 9 * P.N + i;
                float m9[9];
#pragma unroll
                for (int e = 0; e < 9; ++e) m9[e] = __ldg(ms + (int64_t)e * P.N);
                const V* pu = uz + (ty + 2) * PUWE + 3 * (tx + 2);
                const float c0 = in0 ? w0 : 0.f, c1 = in1 ? w1 : 0.f;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float z0 = m9[3 * a] * t0[0] + m9[3 * a + 1] * t0[1] + m9[3 * a + 2] * t0[2];
                    const float z1 = m9[3 * a] * t1[0] + m9[3 * a + 1] * t1[1] + m9[3 * a + 2] * t1[2];
                    const pair_t v = fma2(pk(c0, c1), pk(z0, z1), pu[a]);
                    o[a] = v;
                    if constexpr (EPI) dotp = fma2(rh[a], v, dotp);
                }
            }
        }
    };

    // Tv fills: staged variant a plane ahead at the start of each step; lean variant right after the block barrier
    // that ends the phase 1 reading its single slot.
    bool ok = true;
    if (any_on) {
        if (producer) {
            for (int p = zbeg - 2; p <= zbeg + 1; ++p) issue_u(p);
            issue_tv(zbeg - 1);
            if constexpr (!LEAN) {
                issue_tv(zbeg);
                issue_kn(zbeg);
                if (zbeg + 1 < zend) issue_kn(zbeg + 1);
            }
        }
        wait_planes(zbeg - 2, -1, -1);
        wait_planes(zbeg - 1, zbeg - 1, -1);
        wait_planes(zbeg, -1, -1);
        phase1(zbeg - 1, false, u_slot(zbeg - 2), u_slot(zbeg - 1), u_slot(zbeg), tv_slot(zbeg - 1), nullptr,
               ba_slot(zbeg - 1));
        ok = !__syncthreads_or(lost);
        if (ok) {
            if (producer) {
                fence_proxy_async();
                if (zbeg + 2 <= zend + 1) issue_u(zbeg + 2);
                if constexpr (LEAN)
                    issue_tv(zbeg);
                else if (zbeg + 1 <= zend)
                    issue_tv(zbeg + 1);
            }
            load_kn(zbeg);
            wait_planes(zbeg + 1, zbeg, zbeg);
            phase1(zbeg, true, u_slot(zbeg - 1), u_slot(zbeg), u_slot(zbeg + 1), tv_slot(zbeg), kn_slot(zbeg),
                   ba_slot(zbeg));
            ok = !__syncthreads_or(lost);
            if (LEAN && ok && producer) {
                fence_proxy_async();
                if (zbeg + 1 <= zend) issue_tv(zbeg + 1);
            }
        }
        if (ok) {
            // Slot indices of the z loop, the same for every thread and advanced once per step instead of being
            // recomputed by division at every use.  With s = z - zbeg: the u fill of plane p is number p - (zbeg-2),
            // so plane z-1 sits in slot (s+1) % NUS, and the fill of plane z+2 that this step waits for is number
            // s+4 (parity ((s+4) / NUS) & 1); the Tv fill of plane z+1 is number s+2, the Kn fill number s+1; the
            // (B, A) of plane p sits in slot p mod NBAS.
            auto wrapu = [](int v) { return v >= NUS ? v - NUS : v; };
            auto wrapb = [](int v) { return v >= NBAS ? v - NBAS : v; };
            int iu = 1 % NUS;                               // u slot of plane z-1
            int pu2 = (4 / NUS) & 1;                        // parity of the u fill of plane z+2
            int ib = (((zbeg - 1) % NBAS) + NBAS) % NBAS;   // (B, A) slot of plane z-1
#pragma unroll 2
            for (int z = zbeg, s = 0; z < zend; ++z, ++s) {
                const int iu0 = wrapu(iu + 1), iu1 = wrapu(iu0 + 1), iu2 = wrapu(iu1 + 1);
                const int ib0 = wrapb(ib + 1), ib1 = wrapb(ib0 + 1);
                const int itv = NTV == 2 ? (s & 1) : 0, ptv = NTV == 2 ? (((s + 2) >> 1) & 1) : (s & 1);
                const int ikn = (s + 1) & 1, pkn = ((s + 1) >> 1) & 1;
                const V* uz = su + (size_t)iu0 * US;
#pragma unroll
                for (int a = 0; a < 3; ++a) own_cur[a] = own_next[a];
                if constexpr (!LEAN) {
#pragma unroll
                    for (int k = 0; k < 18; ++k) tv_cur[k] = tv_next[k];
                }
                if (producer) {
                    fence_proxy_async();
                    if (z + 3 <= zend + 1) issue_u(z + 3);
                    if constexpr (!LEAN) {
                        if (z + 2 <= zend) issue_tv(z + 2);
                        if (z + 2 < zend) issue_kn(z + 2);
                    }
                }
                if (z + 1 < zend) load_kn(z + 1);
                if (z + 2 < nz) wait_fill(iu2, pu2);
                if (z + 1 < nz) wait_fill(BTV + itv, ptv);
                if (!LEAN && z + 1 < zend) wait_fill(BKN + ikn, pkn);
                phase1(z + 1, z + 1 < zend, uz, su + (size_t)iu1 * US, su + (size_t)iu2 * US, stv + (size_t)itv * TVS,
                       skn + (size_t)ikn * KNS, sba + (size_t)ib1 * BAS);
                if constexpr (PREF_TV) {
                    if (own_xy) {
                        const CT* tvg = reinterpret_cast<const CT*>(P.Tv) + (int64_t)18 * set * P.N +
                                        ((int64_t)z * ny + gy) * nx + gx;
#pragma unroll
                        for (int k = 0; k < 18; ++k) tv_cur[k] = __ldg(tvg + (int64_t)k * P.N);
                    }
                }
                if (__syncthreads_or(lost)) {  // uniform: every thread leaves the loop at this barrier
                    ok = false;
                    break;
                }
                if (LEAN && producer) {  // the Tv slot is free: fill it with the plane of the next phase 1
                    fence_proxy_async();
                    if (z + 2 <= zend) issue_tv(z + 2);
                }
                phase2(z, sba + (size_t)ib * BAS, sba + (size_t)ib0 * BAS, sba + (size_t)ib1 * BAS, uz);
                // Lean: the next step's Tv fill and phase 1 reuse buffers phase 2 may still read.  Staged: the next
                // step's fills go to the u slot of plane z - 1 and phase 1 writes the (B, A) slot of plane z + 2,
                // neither of which this phase 2 reads, and every warp has left phase 2 of plane z - 1 before any
                // passes this step's barrier: no second barrier.
                if constexpr (LEAN) __syncthreads();
                iu = iu0;
                ib = ib0;
                if (wrapu(iu2 + 1) == 0) pu2 ^= 1;  // the next step waits for fill s+5
            }
        }
        if (!ok && producer) {  // let the copies in flight land before the block's shared memory is released
            for (int b = 0; b < NBAR; ++b)
                if ((pend >> b) & 1u) mbar_wait(&bars[b], (ppar >> b) & 1u);
        }
    }

    if constexpr (EPI) {
        if (!P.part) return;
        CT d0, d1;
        LN::lanes(dotp, d0, d1);
        const int nblk = gridDim.x / P.npp;  // CTAs per system
        for (int j = 0; j < nr; ++j) {
            const int s = sbase + j;
            const double v = block_sum(ok ? (double)(j == 0 ? d0 : d1) : 0.0, red);
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
                    if (P.has_sc) {
                        if constexpr (MODE == PM_DOT)
                            cg_alpha_step(P.scv, s, acc, P.it);
                        else
                            cg_beta_step(P.scv, s, acc, P.it);
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Opt-in to the kernel's dynamic shared memory, once per device (outside any stream capture: pair_prepare).
template <int MODE, bool LEAN, typename CT = float>
cudaError_t pair_attr()
{
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!((attr_set >> dev) & 1ull)) {
        cudaError_t e = cudaFuncSetAttribute(k_sc_pair<MODE, LEAN, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)pair_bytes(LEAN, (int)sizeof(CT)));
        if (e != cudaSuccess) return e;
        attr_set |= 1ull << dev;
    }
    return cudaSuccess;
}

// CT = float: u and out in the pair layout (npair, N, 3, 2); CT = double: natural layout (nsys, N, 3), the FP64
// arrays passed through the float pointers of PairArgs (u, out, Kn, Tv).
template <int MODE, bool LEAN, typename CT = float>
cudaError_t launch_pair(const PairArgs& a, cudaStream_t st)
{
    constexpr int ES = (int)sizeof(CT), NL = PairLane<CT>::NL;
    const int nset = (a.nsys + a.rhs_per_set - 1) / a.rhs_per_set;
    CUtensorMap mu, mtv, mkn;
    {
        // u rows of 3 * NL elements per site; FP64: the systems themselves (a trailing partial set reads zeros)
        const uint64_t nu = NL == 2 ? (uint64_t)a.npair : (uint64_t)a.nsys;
        const uint64_t dims[4] = {(uint64_t)3 * NL * a.nx, (uint64_t)a.ny, (uint64_t)a.nz, nu};
        const uint64_t str[3] = {(uint64_t)3 * NL * a.nx * ES, (uint64_t)3 * NL * a.nx * a.ny * ES,
                                 (uint64_t)3 * NL * a.nx * a.ny * a.nz * ES};
        const uint32_t box[4] = {(uint32_t)(3 * NL * (PX + 4)), (uint32_t)PUH, 1, 1};
        if (!make_tensor_map4(&mu, ES, a.u, dims, str, box)) return cudaErrorInvalidValue;
    }
    {
        const uint64_t dims[4] = {(uint64_t)a.nx, (uint64_t)a.ny, (uint64_t)a.nz, (uint64_t)18 * nset};
        const uint64_t str[3] = {(uint64_t)a.nx * ES, (uint64_t)a.nx * a.ny * ES, (uint64_t)a.nx * a.ny * a.nz * ES};
        const uint32_t btv[4] = {(uint32_t)PTVW, (uint32_t)PSH, 1, 18};
        const uint32_t bkn[4] = {(uint32_t)PKNW, (uint32_t)PY, 1, 18};
        if (!make_tensor_map4(&mtv, ES, a.Tv, dims, str, btv)) return cudaErrorInvalidValue;
        if (LEAN)
            mkn = mtv;  // not read by the lean variant
        else if (!make_tensor_map4(&mkn, ES, a.Kn, dims, str, bkn))
            return cudaErrorInvalidValue;
    }
    cudaError_t e = pair_attr<MODE, LEAN, CT>();
    if (e != cudaSuccess) return e;
    const int ntile = ((a.nx + PX - 1) / PX) * ((a.ny + PY - 1) / PY);
    const int nzc = (a.nz + a.zchunk - 1) / a.zchunk;
    if (a.npair != nset * a.npp || (int64_t)a.npp * ntile * nzc > 0x7FFFFFFF) return cudaErrorInvalidValue;
    for (int s0 = 0; s0 < nset; s0 += 65535) {
        PairArgs b = a;
        b.set0 = s0;
        b.wait_polls = tma_wait_polls();
        const int ns = nset - s0 < 65535 ? nset - s0 : 65535;
        k_sc_pair<MODE, LEAN, CT><<<dim3(a.npp * ntile * nzc, ns), pair_threads(LEAN), pair_bytes(LEAN, ES), st>>>(
            mu, mtv, mkn, b);
    }
    return cudaGetLastError();
}

// (nsys, N, 3) <-> pair layout, one thread per (particle, pair); dummy lanes are written as zero by the packer
__global__ void k_pair_pack(const float* __restrict__ x, float* __restrict__ xp, int64_t N, int nsys, int rps, int npp)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int pr = blockIdx.y, set = pr / npp, jp = pr % npp;
    const int s0 = set * rps + 2 * jp;
    // a trailing partial set leaves pairs (or second lanes) without a system: those lanes are written as zero and
    // nothing past the batch is read
    const bool has0 = s0 < nsys, has1 = 2 * jp + 1 < rps && s0 + 1 < nsys;
    const float* a0 = x + ((int64_t)s0 * N + i) * 3;
    const float* a1 = x + ((int64_t)(s0 + 1) * N + i) * 3;
    pair_t* o = reinterpret_cast<pair_t*>(xp + ((int64_t)pr * N + i) * 6);
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = pk(has0 ? a0[a] : 0.f, has1 ? a1[a] : 0.f);
}

__global__ void k_pair_unpack(const float* __restrict__ xp, float* __restrict__ x, int64_t N, int nsys, int rps,
                              int npp)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int pr = blockIdx.y, set = pr / npp, jp = pr % npp;
    const int s0 = set * rps + 2 * jp;
    if (s0 >= nsys) return;  // a pair of a trailing partial set with no system behind it
    const bool has1 = 2 * jp + 1 < rps && s0 + 1 < nsys;
    const pair_t* v = reinterpret_cast<const pair_t*>(xp + ((int64_t)pr * N + i) * 6);
    float* a0 = x + ((int64_t)s0 * N + i) * 3;
    float* a1 = x + ((int64_t)(s0 + 1) * N + i) * 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float l, h;
        unpk(v[a], l, h);
        a0[a] = l;
        if (has1) a1[a] = h;
    }
}

}  // namespace

cudaError_t pair_pack(const float* x, float* xp, int64_t N, int nsys, int rps, cudaStream_t st)
{
    const int npp = (rps + 1) / 2, nset = (nsys + rps - 1) / rps;
    const int npair = nset * npp;
    if (npair > 65535) return cudaErrorInvalidValue;
    k_pair_pack<<<dim3((unsigned)((N + 255) / 256), npair), 256, 0, st>>>(x, xp, N, nsys, rps, npp);
    return cudaGetLastError();
}

cudaError_t pair_unpack(const float* xp, float* x, int64_t N, int nsys, int rps, cudaStream_t st)
{
    const int npp = (rps + 1) / 2, nset = (nsys + rps - 1) / rps;
    const int npair = nset * npp;
    if (npair > 65535) return cudaErrorInvalidValue;
    k_pair_unpack<<<dim3((unsigned)((N + 255) / 256), npair), 256, 0, st>>>(xp, x, N, nsys, rps, npp);
    return cudaGetLastError();
}

bool pair_supported(int nx) { return nx % 4 == 0 && tma_supported(nx, 4); }

// z planes per CTA: an autotuned value for this shape if one was recorded (lpm_autotune_kmv), else enough z chunks
// for two CTAs per SM of work with at least 8 planes each.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_tuned;  // shape -> (zchunk, variant)
}  // namespace

int pair_zchunk_heuristic(int nx, int ny, int nz, int npair)
{
    const long long base = (long long)((nx + PX - 1) / PX) * ((ny + PY - 1) / PY) * npair;
    int nzc = 1;
    while (base * nzc < 2 * 148 && nz / (nzc + 1) >= 8) ++nzc;
    return (nz + nzc - 1) / nzc;
}

int pair_zchunk(int nx, int ny, int nz, int npair)
{
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tuned.find(std::make_tuple(nx, ny, nz, npair));
        if (it != g_tuned.end()) return it->second.first;
    }
    return pair_zchunk_heuristic(nx, ny, nz, npair);
}

int pair_variant(int nx, int ny, int nz, int npair)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tuned.find(std::make_tuple(nx, ny, nz, npair));
    return it != g_tuned.end() ? it->second.second : kPairDefaultVariant;
}

void pair_zchunk_record(int nx, int ny, int nz, int npair, int zchunk, int variant)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tuned[std::make_tuple(nx, ny, nz, npair)] = std::make_pair(zchunk, variant);
}

int pair_zchunk_max_chunks(int nz) { return nz / 8 > 1 ? nz / 8 : 1; }

int pair_dot_blocks_max(int nx, int ny, int nz) { return ((nx + PX - 1) / PX) * ((ny + PY - 1) / PY) * (nz / 8 + 1); }

cudaError_t launch_sc_pair_mode(const PairArgs& a, int mode, cudaStream_t st)
{
    if (a.npair < 1 || a.npp < 1 || a.zchunk < 1) return cudaErrorInvalidValue;
    if (mode >= PM_RESID && (!a.rhs || !a.fbox || (mode >= PM_SMOOTH && (!a.Ms || !a.fw))))
        return cudaErrorInvalidValue;
    const bool lean = a.variant != 0;
    switch (mode) {
    case PM_NONE: return lean ? launch_pair<PM_NONE, true>(a, st) : launch_pair<PM_NONE, false>(a, st);
    case PM_DOT: return lean ? launch_pair<PM_DOT, true>(a, st) : launch_pair<PM_DOT, false>(a, st);
    case PM_RESID: return lean ? launch_pair<PM_RESID, true>(a, st) : launch_pair<PM_RESID, false>(a, st);
    case PM_SMOOTH: return lean ? launch_pair<PM_SMOOTH, true>(a, st) : launch_pair<PM_SMOOTH, false>(a, st);
    case PM_SMOOTH_DOT:
        return lean ? launch_pair<PM_SMOOTH_DOT, true>(a, st) : launch_pair<PM_SMOOTH_DOT, false>(a, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t pair_prepare()
{
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = pair_attr<PM_NONE, false>();
    if (e == cudaSuccess) e = pair_attr<PM_NONE, true>();
    if (e == cudaSuccess) e = pair_attr<PM_DOT, false>();
    if (e == cudaSuccess) e = pair_attr<PM_DOT, true>();
    if (e == cudaSuccess) e = pair_attr<PM_RESID, false>();
    if (e == cudaSuccess) e = pair_attr<PM_RESID, true>();
    if (e == cudaSuccess) e = pair_attr<PM_SMOOTH, false>();
    if (e == cudaSuccess) e = pair_attr<PM_SMOOTH, true>();
    if (e == cudaSuccess) e = pair_attr<PM_SMOOTH_DOT, false>();
    if (e == cudaSuccess) e = pair_attr<PM_SMOOTH_DOT, true>();
    if (e == cudaSuccess) e = pair_attr<PM_NONE, true, double>();
    if (e == cudaSuccess) e = pair_attr<PM_DOT, true, double>();
    return e;
}

cudaError_t launch_sc_pair(const PairArgs& a, bool epi, cudaStream_t st)
{
    return launch_sc_pair_mode(a, epi ? PM_DOT : PM_NONE, st);
}

bool pair64_supported(int nx) { return nx % 2 == 0 && tma_supported(nx, 8); }

PairArgs pair64_args(int nx, int ny, int nz, int64_t N, int nsys, int rps, const double* u, const double* Kn,
                     const double* Tv, double* out)
{
    PairArgs a{};
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.N = N;
    a.nsys = nsys;
    a.rhs_per_set = rps;
    a.npp = rps;
    a.npair = (nsys + rps - 1) / rps * rps;
    a.zchunk = pair_zchunk_heuristic(nx, ny, nz, a.npair);
    a.variant = 1;
    a.u = reinterpret_cast<const float*>(u);
    a.Kn = reinterpret_cast<const float*>(Kn);
    a.Tv = reinterpret_cast<const float*>(Tv);
    a.out = reinterpret_cast<float*>(out);
    return a;
}

cudaError_t launch_sc_pair64(const PairArgs& a, bool epi, cudaStream_t st)
{
    if (a.npair < 1 || a.npp != a.rhs_per_set || a.zchunk < 1) return cudaErrorInvalidValue;
    return epi ? launch_pair<PM_DOT, true, double>(a, st) : launch_pair<PM_NONE, true, double>(a, st);
}

}  // namespace lpm
