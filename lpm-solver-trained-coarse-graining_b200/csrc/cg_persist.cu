// Persistent batched CG / block-Jacobi PCG: one cooperative launch runs a whole solve.
//
// Same algorithm, stopping rule and freezing as the graph-launched engine of cg.cu (coarse3d/lin3d.py:464-518 with
// the batching of coarse3d/torch_lpm3d.py:109-140).  On small lattices an iteration of that engine is four short
// kernels whose launch gaps, plus a host poll every few iterations, cost more than their work; here every iteration
// of every system runs inside one kernel and the host waits once.
//
// Teams.  The grid is split into `nteam` teams of B blocks.  Team t owns systems t, t + nteam, t + 2 nteam, ...
// with all of their particles, so the operator's neighbourhoods, the inner products and the scalar steps of a
// system never leave its team: the phases of an iteration are separated by team barriers (one monotonic arrival
// counter per team; with B = 1 a block barrier) rather than grid-wide ones.  Every block of a team sums the team's
// per-block partials in the same fixed order, so all blocks compute the same alpha, beta, convergence test and
// freezing without another barrier; the team's first block writes the caller's outputs.
//
// One iteration, three barriers (z = r for plain CG):
//   A  p' = z + beta p for the block's particles (into the other p buffer) and the shell sums of p' (neighbours'
//      p' recomputed from their z and p), into st                                                  | barrier
//   B  Ap = mask(K p') from st; p'.Ap partials                                                     | barrier
//   C  alpha = r.z / p'.Ap;  x += alpha p';  r -= alpha Ap;  z = mask(M r);  r.z, r.r partials     | barrier
//   then beta = r.z_new / r.z, the convergence test every `check` iterations and the freezing of converged systems.
// The first iteration runs with beta = 0 and p = 0, i.e. p' = z.
//
// Co-residency.  The launch is cooperative, so all blocks are resident together; cooperative launches of this
// library are chained on the device by an event, so two persistent solves never hold the GPU's slots at the same
// time (blocks of ordinary kernels only delay a launch).  Every barrier wait is bounded in time: on expiry a block
// records LPM_ERR_TIMEOUT and returns, and the blocks waiting on it see the code and return too.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <type_traits>

#include "lpm_cg.h"
#include "lpm_sqtile.cuh"
#include "lpm_stencil.cuh"

namespace lpm {

namespace {

using namespace stencil;

constexpr int PB = 256;        // threads per block
constexpr int MAXST = 16;      // systems per team
constexpr unsigned long long WAIT_NS = 2000000000ull;  // default bound of one barrier wait (2 s)
std::atomic<unsigned long long> g_wait_ns{WAIT_NS};     // current bound (lpm_set_wait_limit_ns)

template <typename T>
struct PersistArgs {
    int nx, ny, nz;
    int64_t N;
    CoefLayout cl;
    Batch bt;
    const T *Kn, *Tv, *Minv;
    const uint8_t* mask;
    const T* b;
    const T* Ax;  // K x of a nonzero start, or null
    T* x;
    T *r, *z, *p0, *p1, *Ap, *st;
    double* part;   // (4, nsys, B): p'.Ap, r.z, r.r, b.b per block
    unsigned* bar;  // (nteam) arrival counters, zero at launch
    int* err;
    unsigned long long wait_ns;  // bound of one team-barrier wait
    int* iters;
    double* relres;
    int* status;
    const double* tols;
    int nteam, B, check, maxit, precheck;
    double tol;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Team barrier number `n` (1, 2, ...): every block adds one arrival; the barrier is passed when the counter reaches
// n * B.  Returns false when the wait expired or another block of the grid reported an error.
__device__ __forceinline__ bool team_sync(unsigned* ctr, unsigned n, int B, int* err, int* s_abort,
                                          unsigned long long wait_ns)
{
    __syncthreads();
    if (B > 1 && threadIdx.x == 0) {
        // arrive with release semantics (the block's writes, ordered before by the block barrier, become visible
        // first); the acquiring load below orders the block's later reads after the other blocks' writes
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" : : "l"(ctr), "r"(1u) : "memory");
        const unsigned target = n * (unsigned)B;
        const unsigned long long t0 = global_ns();
        for (unsigned polls = 0; (int)(ld_acquire(ctr) - target) < 0; ++polls) {
            if (*(volatile int*)err != 0) {
                *s_abort = 1;
                break;
            }
            if (global_ns() - t0 >= wait_ns) {  // wait_ns = 0: expire unless the barrier is passed at once
                atomicCAS(err, 0, LPM_ERR_TIMEOUT);
                *s_abort = 1;
                break;
            }
            if (polls > 64) __nanosleep(32);
        }
    }
    __syncthreads();
    return *s_abort == 0;
}

template <typename T, int DIM>
__device__ __forceinline__ void block_mv(const T* __restrict__ M, const T* r, T* z)
{
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        T acc = 0;
#pragma unroll
        for (int b = 0; b < DIM; ++b) acc += M[a * DIM + b] * r[b];
        z[a] = acc;
    }
}

// Coordinates of particle i of a full box (the engine takes boxes of fewer than 2^31 particles).
template <class NB>
__device__ __forceinline__ Site site_at(int nx, int ny, int64_t i, int s)
{
    Site p;
    p.i = i;
    p.s = s;
    p.ok = true;
    if constexpr (NB::structured) {
        const unsigned ii = (unsigned)i, row = ii / (unsigned)nx;
        p.x = (int)(ii - row * (unsigned)nx);
        p.y = (int)(row % (unsigned)ny);
        p.z = (int)(row / (unsigned)ny);
    } else {
        p.x = p.y = p.z = 0;
    }
    return p;
}

// Team totals of value v for the block's systems (those with on[js] set): warp w takes systems w, w + 8, ...; lane l
// sums the partials of blocks l, l + 32, ... in order, then a fixed shuffle tree, so every block of the team gets
// bit-identical totals.
__device__ __forceinline__ void team_totals(const double* part, int v, int nsys, int B, int team, int nteam, int nst,
                                            const int* on, double* out)
{
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (int js = w; js < nst; js += PB / 32) {
        if (on && !on[js]) continue;
        const double* row = part + ((int64_t)v * nsys + team + js * nteam) * B;
        double acc = 0.0;
        for (int k = l; k < B; k += 32) acc += __ldcg(row + k);
        acc = warp_sum(acc);
        if (l == 0) out[js] = acc;
    }
}

template <typename T, int DIM, class NB, bool PREC>
__global__ void __launch_bounds__(PB) k_cg_persist(NB nb, PersistArgs<T> a)
{
    // full 2D boxes: the operator's two passes on shared-memory tiles, two barriers per iteration
    constexpr bool FUSED2D = DIM == 2 && NB::structured;
    __shared__ std::conditional_t<FUSED2D, sqtile::Smem<T>, char> tsm;
    __shared__ double sh[32];
    __shared__ double s_rz[MAXST], s_bn[MAXST], s_beta[MAXST], s_alpha[MAXST], s_pap[MAXST];
    __shared__ double s_t[3][MAXST];  // team totals
    __shared__ int s_act[MAXST];
    __shared__ int s_abort;
    const int team = blockIdx.x / a.B, rb = blockIdx.x % a.B;
    const int nsys = a.bt.nsys;
    const int nst = team < nsys ? (nsys - team + a.nteam - 1) / a.nteam : 0;
    const int64_t N = a.N;
    // this block's particle range of every system of the team
    const int64_t chunk = (N + a.B - 1) / a.B;
    const int64_t lo = (int64_t)rb * chunk, hi = lo + chunk < N ? lo + chunk : N;
    unsigned* ctr = a.bar + team;
    unsigned nbar = 0;
    if (threadIdx.x == 0) s_abort = 0;
    __syncthreads();

    auto sys_of = [&](int js) { return team + js * a.nteam; };
    auto free_dof = [&](int s, int64_t i, int c) {
        return a.mask == nullptr || a.mask[((int64_t)(s % a.bt.nmask) * N + i) * DIM + c] != 0;
    };
    // block partial of value v for system s (every thread passes its sum; block_sum synchronises)
    auto put_partial = [&](double val, int v, int s) {
        const double t = block_sum(val, sh);
        if (threadIdx.x == 0) a.part[((int64_t)v * nsys + s) * a.B + rb] = t;
    };

    // ------------------------------------------------------------------------------------------------ start
    for (int js = 0; js < nst; ++js) {
        const int s = sys_of(js);
        double v[3] = {0.0, 0.0, 0.0};  // b.b, r.z, r.r
        for (int64_t i = lo + threadIdx.x; i < hi; i += PB) {
            const int64_t o = ((int64_t)s * N + i) * DIM;
            T rv[DIM], zv[DIM];
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                const T bv = a.b[o + c];
                T w = a.Ax ? bv - a.Ax[o + c] : bv;
                if (!free_dof(s, i, c)) w = T(0);
                rv[c] = w;
                v[0] += (double)bv * (double)bv;
            }
            if constexpr (PREC) {
                block_mv<T, DIM>(a.Minv + ((int64_t)(s / a.bt.rhs_per_set) * N + i) * DIM * DIM, rv, zv);
#pragma unroll
                for (int c = 0; c < DIM; ++c)
                    if (!free_dof(s, i, c)) zv[c] = T(0);
            } else {
#pragma unroll
                for (int c = 0; c < DIM; ++c) zv[c] = rv[c];
            }
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
                a.r[o + c] = rv[c];
                if constexpr (PREC) a.z[o + c] = zv[c];
                a.p0[o + c] = T(0);
                v[1] += (double)rv[c] * (double)zv[c];
                v[2] += (double)rv[c] * (double)rv[c];
            }
        }
        put_partial(v[0], 3, s);
        put_partial(v[1], 1, s);
        put_partial(v[2], 2, s);
    }
    if (!team_sync(ctr, ++nbar, a.B, a.err, &s_abort, a.wait_ns)) return;
    team_totals(a.part, 3, nsys, a.B, team, a.nteam, nst, nullptr, s_t[0]);
    team_totals(a.part, 1, nsys, a.B, team, a.nteam, nst, nullptr, s_t[1]);
    team_totals(a.part, 2, nsys, a.B, team, a.nteam, nst, nullptr, s_t[2]);
    __syncthreads();
    if (threadIdx.x < nst) {
        const int js = threadIdx.x, s = sys_of(js);
        const double bb = s_t[0][js], rz = s_t[1][js], rr = s_t[2][js];
        const double bn = sqrt(bb);
        const double rel = bn > 0.0 ? sqrt(rr) / bn : 0.0;
        const bool finite = isfinite(bn) && isfinite(rz) && isfinite(rr);
        int act = bn > 0.0 && finite;
        if (act && a.precheck && rel <= (a.tols ? a.tols[s] : a.tol)) act = 0;
        s_bn[js] = bn;
        s_rz[js] = rz;
        s_beta[js] = 0.0;
        s_act[js] = act;
        if (rb == 0) {
            a.iters[s] = 0;
            a.relres[s] = rel;
            a.status[s] = finite ? LPM_STATUS_OK : LPM_STATUS_BREAKDOWN;
        }
    }
    __syncthreads();

    const T* zsrc = PREC ? a.z : a.r;
    for (int it = 1; it <= a.maxit; ++it) {
        int any = 0;
        for (int js = 0; js < nst; ++js) any |= s_act[js];
        if (!any) break;
        T* pc = (it & 1) ? a.p0 : a.p1;  // p of the previous iteration
        T* pn = (it & 1) ? a.p1 : a.p0;  // p' of this one

        if constexpr (FUSED2D) {
            // ------------------------------------------------------- A+B: p', K p' and p'.Ap on 2D tiles
            const int ntx = sqtile::tiles_x(a.nx), ntile = ntx * sqtile::tiles_y(a.ny);
            for (int js = 0; js < nst; ++js) {
                if (!s_act[js]) continue;
                const int s = sys_of(js);
                const T be = (T)s_beta[js];
                const T* zs = zsrc + (int64_t)s * N * 2;
                const T* ps = pc + (int64_t)s * N * 2;
                T* pns = pn + (int64_t)s * N * 2;
                const int64_t cbase = (int64_t)(s / a.bt.rhs_per_set) * a.cl.set_stride;
                auto load = [&](int64_t q, T* v) {
                    v[0] = zs[2 * q] + be * ps[2 * q];
                    v[1] = zs[2 * q + 1] + be * ps[2 * q + 1];
                };
                double dot = 0.0;
                for (int t = rb; t < ntile; t += a.B) {
                    const int x0 = (t % ntx) * sqtile::TX, y0 = (t / ntx) * sqtile::TY;
                    const sqtile::GlobalCoef<T> kn{a.Kn + cbase, a.cl, a.nx, x0, y0};
                    const sqtile::GlobalCoef<T> tv{a.Tv + cbase, a.cl, a.nx, x0, y0};
                    sqtile::stage(a.nx, a.ny, x0, y0, load, tsm);
                    __syncthreads();
                    sqtile::sums(a.nx, a.ny, x0, y0, tv, tsm);
                    __syncthreads();
                    sqtile::forces(a.nx, a.ny, x0, y0, kn, tv, tsm,
                                   [&](int64_t i, T (&f)[2], const T* ui) {
                                       pns[2 * i] = ui[0];
                                       pns[2 * i + 1] = ui[1];
                                       T* o = a.Ap + ((int64_t)s * N + i) * 2;
#pragma unroll
                                       for (int c = 0; c < 2; ++c) {
                                           if (!free_dof(s, i, c)) f[c] = T(0);
                                           o[c] = f[c];
                                           dot += (double)ui[c] * (double)f[c];
                                       }
                                   });
                    __syncthreads();
                }
                put_partial(dot, 0, s);
            }
        } else {
            // -------------------------------------------------------------------------------- A: p' and shell sums
            for (int js = 0; js < nst; ++js) {
                if (!s_act[js]) continue;
                const int s = sys_of(js);
                const T be = (T)s_beta[js];
                const T* zs = zsrc + (int64_t)s * N * DIM;
                const T* ps = pc + (int64_t)s * N * DIM;
                T* pns = pn + (int64_t)s * N * DIM;
                const T* tvs = a.Tv + (int64_t)(s / a.bt.rhs_per_set) * a.cl.set_stride;
                auto load = [&](int64_t q, T* uq) {
#pragma unroll
                    for (int c = 0; c < DIM; ++c) uq[c] = zs[DIM * q + c] + be * ps[DIM * q + c];
                };
                for (int64_t i = lo + threadIdx.x; i < hi; i += PB) {
                    const Site p = site_at<NB>(a.nx, a.ny, i, s);
                    T ui[3];
                    load(i, ui);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) pns[DIM * i + c] = ui[c];
                    T o4[4];
                    shell_sums_at<T, DIM>(nb, p, ui, load, tvs + i * a.cl.site_stride, a.cl.slot_stride, o4);
                    T* o = a.st + ((int64_t)s * N + i) * 4;
#pragma unroll
                    for (int c = 0; c < 4; ++c) o[c] = o4[c];
                }
            }
            if (!team_sync(ctr, ++nbar, a.B, a.err, &s_abort, a.wait_ns)) return;

            // ------------------------------------------------------------------------------------- B: Ap, p'.Ap
            for (int js = 0; js < nst; ++js) {
                if (!s_act[js]) continue;
                const int s = sys_of(js);
                const T* us = pn + (int64_t)s * N * DIM;
                const T* sts = a.st + (int64_t)s * N * 4;
                const int64_t cbase = (int64_t)(s / a.bt.rhs_per_set) * a.cl.set_stride;
                auto load = [&](int64_t q, T* uq) {
#pragma unroll
                    for (int c = 0; c < DIM; ++c) uq[c] = us[DIM * q + c];
                };
                auto sums = [&](int64_t q, T (&Sq)[2], T (&TSq)[2]) {
                    load4(sts + 4 * q, Sq[0], Sq[1], TSq[0], TSq[1]);
                };
                double dot = 0.0;
                for (int64_t i = lo + threadIdx.x; i < hi; i += PB) {
                    const Site p = site_at<NB>(a.nx, a.ny, i, s);
                    T ui[3];
                    load(i, ui);
                    T Si[2], TSi[2];
                    sums(i, Si, TSi);
                    T f[3];
                    force_at<T, DIM>(nb, p, ui, load, sums, Si, TSi, a.Kn + cbase + i * a.cl.site_stride,
                                     a.Tv + cbase + i * a.cl.site_stride, a.Kn + cbase, a.Tv + cbase, a.cl, f);
                    T* o = a.Ap + ((int64_t)s * N + i) * DIM;
#pragma unroll
                    for (int c = 0; c < DIM; ++c) {
                        if (!free_dof(s, i, c)) f[c] = T(0);
                        o[c] = f[c];
                        dot += (double)ui[c] * (double)f[c];
                    }
                }
                put_partial(dot, 0, s);
            }
        }
        if (!team_sync(ctr, ++nbar, a.B, a.err, &s_abort, a.wait_ns)) return;
        team_totals(a.part, 0, nsys, a.B, team, a.nteam, nst, s_act, s_t[0]);
        __syncthreads();
        if (threadIdx.x < nst && s_act[threadIdx.x]) {
            const int js = threadIdx.x;
            const double pAp = s_t[0][js];
            const double rzc = s_rz[js];
            const bool good = pAp > 0.0 && isfinite(pAp) && isfinite(rzc);
            s_pap[js] = pAp;
            s_alpha[js] = good ? rzc / pAp : 0.0;
        }
        __syncthreads();

        // ----------------------------------------------------------------------- C: x, r, z updates, r.z, r.r
        for (int js = 0; js < nst; ++js) {
            if (!s_act[js]) continue;
            const int s = sys_of(js);
            const T al = (T)s_alpha[js];
            double v[2] = {0.0, 0.0};
            for (int64_t i = lo + threadIdx.x; i < hi; i += PB) {
                const int64_t o = ((int64_t)s * N + i) * DIM;
                T rv[DIM], zv[DIM];
#pragma unroll
                for (int c = 0; c < DIM; ++c) {
                    a.x[o + c] += al * pn[o + c];
                    rv[c] = a.r[o + c] - al * a.Ap[o + c];
                    a.r[o + c] = rv[c];
                }
                if constexpr (PREC) {
                    block_mv<T, DIM>(a.Minv + ((int64_t)(s / a.bt.rhs_per_set) * N + i) * DIM * DIM, rv, zv);
#pragma unroll
                    for (int c = 0; c < DIM; ++c) {
                        if (!free_dof(s, i, c)) zv[c] = T(0);
                        a.z[o + c] = zv[c];
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < DIM; ++c) zv[c] = rv[c];
                }
#pragma unroll
                for (int c = 0; c < DIM; ++c) {
                    v[0] += (double)rv[c] * (double)zv[c];
                    v[1] += (double)rv[c] * (double)rv[c];
                }
            }
            put_partial(v[0], 1, s);
            put_partial(v[1], 2, s);
        }
        if (!team_sync(ctr, ++nbar, a.B, a.err, &s_abort, a.wait_ns)) return;
        team_totals(a.part, 1, nsys, a.B, team, a.nteam, nst, s_act, s_t[1]);
        team_totals(a.part, 2, nsys, a.B, team, a.nteam, nst, s_act, s_t[2]);
        __syncthreads();
        if (threadIdx.x < nst && s_act[threadIdx.x]) {
            const int js = threadIdx.x, s = sys_of(js);
            const double rzn = s_t[1][js], rrn = s_t[2][js];
            const double rzc = s_rz[js], pAp = s_pap[js];
            const double rel = sqrt(rrn) / s_bn[js];
            const double tl = a.tols ? a.tols[s] : a.tol;
            s_beta[js] = rzc != 0.0 ? rzn / rzc : 0.0;
            s_rz[js] = rzn;
            if (!isfinite(pAp) || pAp < 0.0 || !isfinite(rrn) || !isfinite(rzn)) {
                s_act[js] = 0;
                if (rb == 0) {
                    a.iters[s] = it;
                    a.relres[s] = rel;
                    a.status[s] = LPM_STATUS_BREAKDOWN;
                }
            } else if (it % a.check == 0 || it == a.maxit) {
                if (rb == 0) a.relres[s] = rel;
                if (rel <= tl || it == a.maxit) {
                    s_act[js] = 0;
                    if (rb == 0) {
                        a.iters[s] = it;
                        if (rel > tl) a.status[s] = LPM_STATUS_NOT_CONVERGED;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------- host side
inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

struct Carve {
    char* base;
    size_t off;
    template <typename X>
    X* take(size_t count)
    {
        X* p = base ? reinterpret_cast<X*>(base + off) : nullptr;
        off = align_up(off + count * sizeof(X));
        return p;
    }
};

// Largest grid of this kernel that is resident at once (blocks per SM x SMs), per device.
template <typename T, int DIM, class NB, bool PREC>
int resident_blocks()
{
    static std::mutex mu;
    static std::map<int, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_persist<T, DIM, NB, PREC>, PB, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    const int n = coop ? per_sm * sms : 0;
    cache[dev] = n;
    return n;
}

// Serialise this library's cooperative launches on a device: each one waits (on the device) for the previous.
class CoopChain {
  public:
    cudaError_t before(cudaStream_t st, int dev)
    {
        mu_.lock();
        cudaEvent_t& ev = ev_[dev];
        if (ev == nullptr) {
            cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) {
                mu_.unlock();
                return e;
            }
            return cudaSuccess;
        }
        cudaError_t e = cudaStreamWaitEvent(st, ev, 0);
        if (e != cudaSuccess) mu_.unlock();
        return e;
    }
    cudaError_t after(cudaStream_t st, int dev)
    {
        cudaError_t e = cudaEventRecord(ev_[dev], st);
        mu_.unlock();
        return e;
    }

  private:
    std::mutex mu_;
    std::map<int, cudaEvent_t> ev_;
};

CoopChain& coop_chain()
{
    static CoopChain c;
    return c;
}

// Blocks per team never exceed one per PB particles, so partials sized for that bound fit every team shape.
inline int max_team_blocks(int64_t N) { return (int)std::max<int64_t>(1, (N + PB - 1) / PB); }

struct TeamShape {
    int nteam, B;
};

// Teams for nsys systems of N particles on `res` resident blocks: one team per system while they fit (at most
// MAXST systems per team), each team as many blocks as the resident grid allows, up to one particle per thread (a
// 2D tile per block): the phases are latency-bound, so spreading a system wider shortens them.
TeamShape team_shape(int nsys, int64_t N, int res)
{
    TeamShape t{0, 0};
    if (res < 1 || nsys < 1) return t;
    const int nteam = std::min(nsys, res);
    if ((nsys + nteam - 1) / nteam > MAXST) return t;
    t.nteam = nteam;
    t.B = std::max(1, std::min(res / nteam, max_team_blocks(N)));
    return t;
}

template <typename T>
size_t persist_bytes(const Lattice& L, const Batch& bt, int B)
{
    Carve cv{nullptr, 0};
    const size_t nv = (size_t)bt.nsys * L.N * L.dim;
    for (int k = 0; k < 5; ++k) cv.take<T>(nv);  // r, z, p0, p1, Ap
    cv.take<T>((size_t)bt.nsys * L.N * 4);        // st
    cv.take<double>((size_t)4 * bt.nsys * std::max(B, 1));
    cv.take<unsigned>(bt.nsys);
    cv.take<int>(1);
    return cv.off + 256;
}

template <typename T, int DIM, class NB, bool PREC>
int run_persist(NB nb, const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                const T* Minv, const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o, void* ws,
                size_t ws_bytes, int* iters, double* relres, int* status, cudaStream_t st)
{
    const TeamShape ts = team_shape(bt.nsys, L.N, resident_blocks<T, DIM, NB, PREC>());
    if (ts.nteam == 0) return LPM_ERR_ARG;
    char* base = static_cast<char*>(ws);
    const size_t shift = (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    Carve cv{base + shift, 0};
    PersistArgs<T> a{};
    const size_t nv = (size_t)bt.nsys * L.N * L.dim;
    a.r = cv.take<T>(nv);
    a.z = cv.take<T>(nv);
    a.p0 = cv.take<T>(nv);
    a.p1 = cv.take<T>(nv);
    a.Ap = cv.take<T>(nv);
    a.st = cv.take<T>((size_t)bt.nsys * L.N * 4);
    a.part = cv.take<double>((size_t)4 * bt.nsys * ts.B);
    a.bar = cv.take<unsigned>(bt.nsys);
    a.err = cv.take<int>(1);
    if (cv.off + shift > ws_bytes) return LPM_ERR_WORKSPACE;
    a.nx = L.nx;
    a.ny = L.ny;
    a.nz = L.nz;
    a.N = L.N;
    a.cl = cl;
    a.bt = bt;
    a.Kn = Kn;
    a.Tv = Tv;
    a.Minv = Minv;
    a.mask = mask;
    a.b = b;
    a.x = x;
    a.iters = iters;
    a.relres = relres;
    a.status = status;
    a.tols = o.tol_sys;
    a.nteam = ts.nteam;
    a.B = ts.B;
    a.check = o.check;
    a.maxit = o.maxit;
    a.precheck = o.precheck;
    a.tol = o.tol;
    a.wait_ns = g_wait_ns.load();
    cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned) * bt.nsys, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.err, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
    if (!x_is_zero) {
        // K x of the start into Ap (the kernel reads it before its first operator phase)
        if ((e = launch_kmv<T>(L, x, Kn, Tv, cl, bt, a.Ap, a.st, nullptr, st)) != cudaSuccess) return (int)e;
        a.Ax = a.Ap;
    }
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return (int)e;
    CoopChain& ch = coop_chain();
    if ((e = ch.before(st, dev)) != cudaSuccess) return (int)e;
    void* args[] = {&nb, &a};
    e = cudaLaunchCooperativeKernel((const void*)k_cg_persist<T, DIM, NB, PREC>, dim3(ts.nteam * ts.B), dim3(PB),
                                    args, 0, st);
    const cudaError_t e2 = ch.after(st, dev);
    if (e != cudaSuccess) return (int)e;
    if (e2 != cudaSuccess) return (int)e2;
    int err = 0;
    e = cudaMemcpyAsync(&err, a.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return (int)e;
    return err ? err : LPM_OK;
}

template <typename T, int DIM, class NB>
int dispatch_prec(NB nb, const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                  const T* Minv, const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o,
                  void* ws, size_t ws_bytes, int* iters, double* relres, int* status, cudaStream_t st)
{
    if (Minv)
        return run_persist<T, DIM, NB, true>(nb, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws, ws_bytes,
                                             iters, relres, status, st);
    return run_persist<T, DIM, NB, false>(nb, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws, ws_bytes, iters,
                                          relres, status, st);
}

}  // namespace

bool persist_fits(const Lattice& L, const Batch& bt)
{
    if (L.N < 1 || bt.nsys < 1) return false;
    int dev = 0, sms = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) || !coop)
        return false;
    // one resident block per SM is the least any instance gets, so the team shape exists for every instance
    return team_shape(bt.nsys, L.N, sms).nteam > 0;
}

// The automatic choice: 2D batches of up to 2^17 particle-systems (the precision is kept in the interface; both
// thresholds are 2^17 today).  Plain CG per iteration on one B200, packed coefficients, persistent vs launched (the
// launched operator forming the p-update): FP64 15.0 vs 21.5 us at 4 x 128^2, 31.7 vs 24.8 at 10 x 128^2, 132 vs 86
// at 40 x 128^2; FP32 14.5 vs 18.7 at 4 x 128^2, 24.7 vs 23.9 at 10 x 128^2, 23.8 vs 20.8 at 40 x 64^2.  A
// persistent block takes its team's tiles one after another, while the launched operator has every tile of the
// batch in flight.  (3D: the operator's fused TMA kernels are faster than the persistent kernel's
// per-particle passes at every size measured.)
bool persist_auto(const Lattice& L, const Batch& bt, int elem_bytes)
{
    const int64_t units = (int64_t)bt.nsys * L.N;
    (void)elem_bytes;
    const int64_t cap = (int64_t)1 << 17;
    return L.dim == 2 && units <= cap && persist_fits(L, bt);
}

size_t persist_workspace_bytes(const Lattice& L, const Batch& bt, int elem_bytes)
{
    const int B = max_team_blocks(L.N);
    return elem_bytes == 4 ? persist_bytes<float>(L, bt, B) : persist_bytes<double>(L, bt, B);
}

template <typename T>
int cg_solve_persist(const Lattice& L, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                     const T* Minv, const uint8_t* mask, const T* b, T* x, int x_is_zero, const lpm_cg_opts& o,
                     void* ws, size_t ws_bytes, int* iters, double* relres, int* status, cudaStream_t st)
{
    if (o.maxit < 0 || o.check < 1 || bt.nsys < 1) return LPM_ERR_ARG;
    if (L.dim == 3) {
        if (L.nbr)
            return dispatch_prec<T, 3>(TableNb<3>{L.nbr}, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws,
                                       ws_bytes, iters, relres, status, st);
        return dispatch_prec<T, 3>(GridNb<3>{L.nx, L.ny, L.nz}, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws,
                                   ws_bytes, iters, relres, status, st);
    }
    if (L.nbr)
        return dispatch_prec<T, 2>(TableNb<2>{L.nbr}, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws, ws_bytes,
                                   iters, relres, status, st);
    return dispatch_prec<T, 2>(GridNb<2>{L.nx, L.ny, 1}, L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, o, ws,
                               ws_bytes, iters, relres, status, st);
}

unsigned long long persist_wait_limit(unsigned long long ns) { return g_wait_ns.exchange(ns); }

template int cg_solve_persist<float>(const Lattice&, const float*, const float*, const CoefLayout&, const Batch&,
                                     const float*, const uint8_t*, const float*, float*, int, const lpm_cg_opts&,
                                     void*, size_t, int*, double*, int*, cudaStream_t);
template int cg_solve_persist<double>(const Lattice&, const double*, const double*, const CoefLayout&, const Batch&,
                                      const double*, const uint8_t*, const double*, double*, int, const lpm_cg_opts&,
                                      void*, size_t, int*, double*, int*, cudaStream_t);

}  // namespace lpm
