// extern "C" entry points of liblpm_b200.so (declared in include/lpm_b200.h).
#include <cstdint>

#include "../../include/lpm_b200.h"
#include "lpm_amg.h"
#include "lpm_cg.h"
#include "lpm_tma.h"
#include "lpm_kernels.h"
#include "lpm_graph.h"
#include "lpm_abi.h"

using namespace lpm;

namespace {

inline cudaStream_t S(void* p) { return static_cast<cudaStream_t>(p); }

// Scratch handed to kernels is re-aligned to 256 bytes (vector loads of the shell sums need 16/32-byte alignment).
template <typename T>
T* aligned(void* p, size_t bytes, size_t need, int& rc)
{
    const size_t shift = (256 - (reinterpret_cast<uintptr_t>(p) & 255)) & 255;
    if (!p || bytes < need + shift) {
        rc = LPM_ERR_WORKSPACE;
        return nullptr;
    }
    rc = LPM_OK;
    return reinterpret_cast<T*>(static_cast<char*>(p) + shift);
}

inline int ret(cudaError_t e) { return e == cudaSuccess ? LPM_OK : (int)e; }

template <typename T>
int kmv_impl(int dim, const lpm_lattice* lat, const T* u, const T* Kn, const T* Tv, int32_t layout,
             const lpm_batch* batch, T* out, void* scratch, size_t scratch_bytes, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc) return rc;
    if (L.dim != dim) return LPM_ERR_UNSUPPORTED;
    if ((rc = to_batch(batch, bt)) || (rc = to_layout(layout, L, cl))) return rc;
    if (!u || !Kn || !Tv || !out) return LPM_ERR_ARG;
    if constexpr (sizeof(T) == 4) {
        if (dim == 3 && !L.nbr && layout == LPM_LAYOUT_SOA && pair_supported(L.nx) && tma_aligned(u, Kn, Tv)) {
            // full SC box, packed FP32 coefficients: pair-packed operator on pair-layout copies in the scratch
            const int npp = (bt.rhs_per_set + 1) / 2, nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
            const size_t nvp = (size_t)nset * npp * L.N * 6;
            float* up = aligned<float>(scratch, scratch_bytes, 2 * nvp * sizeof(float), rc);
            if (rc) return rc;
            if (nset * npp > 65535) return LPM_ERR_UNSUPPORTED;
            PairArgs a{};
            a.nx = L.nx;
            a.ny = L.ny;
            a.nz = L.nz;
            a.N = L.N;
            a.nsys = bt.nsys;
            a.rhs_per_set = bt.rhs_per_set;
            a.npp = npp;
            a.npair = nset * npp;
            a.zchunk = pair_zchunk(L.nx, L.ny, L.nz, a.npair);
            a.variant = pair_variant(L.nx, L.ny, L.nz, a.npair);
            a.u = up;
            a.Kn = Kn;
            a.Tv = Tv;
            a.out = up + nvp;
            cudaError_t e = pair_pack(u, up, L.N, bt.nsys, bt.rhs_per_set, S(stream));
            if (e == cudaSuccess) e = launch_sc_pair(a, false, S(stream));
            if (e == cudaSuccess) e = pair_unpack(up + nvp, out, L.N, bt.nsys, bt.rhs_per_set, S(stream));
            return ret(e);
        }
    }
    if constexpr (sizeof(T) == 8) {
        if (dim == 3 && !L.nbr && layout == LPM_LAYOUT_SOA && pair64_supported(L.nx) && tma_aligned(u, Kn, Tv)) {
            // full SC box, packed FP64 coefficients: the FP64 instantiation of the pair operator (no scratch)
            const PairArgs a = pair64_args(L.nx, L.ny, L.nz, L.N, bt.nsys, bt.rhs_per_set, u, Kn, Tv, out);
            return ret(launch_sc_pair64(a, false, S(stream)));
        }
    }
    if (dim == 3 && !L.nbr && layout == LPM_LAYOUT_SOA && tma_supported(L.nx, (int)sizeof(T)) &&
        tma_aligned(u, Kn, Tv)) {
        // full SC box with packed coefficients: TMA-fed single-pass operator (needs no scratch)
        TmaArgs<T> a{};
        a.nx = L.nx;
        a.ny = L.ny;
        a.nz = L.nz;
        a.N = L.N;
        a.nsys = bt.nsys;
        a.rhs_per_set = bt.rhs_per_set;
        a.nmask = bt.nmask;
        tma_configure(a);
        a.u = u;
        a.Kn = Kn;
        a.Tv = Tv;
        a.out = out;
        return ret(launch_sc_tma<T>(a, false, S(stream)));
    }
    T* st = aligned<T>(scratch, scratch_bytes, (size_t)bt.nsys * L.N * 4 * sizeof(T), rc);
    if (rc) return rc;
    return ret(launch_kmv<T>(L, u, Kn, Tv, cl, bt, out, st, nullptr, S(stream)));
}

template <typename T>
int cg_impl(const lpm_lattice* lat, const T* Kn, const T* Tv, int32_t layout, const lpm_batch* batch, const T* Minv,
            const uint8_t* mask, const T* b, T* x, int32_t x_is_zero, const lpm_cg_opts* opts, void* ws,
            size_t ws_bytes, int32_t* iters, double* relres, int32_t* status, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(layout, L, cl))) return rc;
    if (!Kn || !Tv || !b || !x || !opts || !ws || !iters || !relres || !status) return LPM_ERR_ARG;
    if (!(opts->tol >= 0.0)) return LPM_ERR_ARG;
    return cg_solve<T>(L, Kn, Tv, cl, bt, Minv, mask, b, x, x_is_zero, *opts, ws, ws_bytes, iters, relres, status,
                       S(stream));
}

}  // namespace

extern "C" {

int lpm_abi_version(void) { return LPM_ABI_VERSION; }

uint64_t lpm_set_wait_limit_ns(uint64_t ns) { return (uint64_t)persist_wait_limit((unsigned long long)ns); }

uint32_t lpm_set_tma_wait_polls(uint32_t polls) { return tma_set_wait_polls(polls); }

void lpm_graph_stats(int64_t* captures, int64_t* entries, int64_t* flushes)
{
    long long c = 0, e = 0, f = 0;
    lpm::graph_stats(&c, &e, &f);
    if (captures) *captures = c;
    if (entries) *entries = e;
    if (flushes) *flushes = f;
}

const char* lpm_status_string(int code)
{
    switch (code) {
    case LPM_OK: return "ok";
    case LPM_ERR_ARG: return "invalid argument";
    case LPM_ERR_WORKSPACE: return "workspace or scratch buffer too small";
    case LPM_ERR_UNSUPPORTED: return "unsupported lattice or precision for this entry point";
    case LPM_ERR_TIMEOUT: return "a bounded device-side wait expired";
    default: return code > 0 ? cudaGetErrorString((cudaError_t)code) : "unknown error";
    }
}

int lpm_pack_coef_f32(const double* src, float* dst, int64_t n, int32_t slots, int32_t nset, void* stream)
{
    if (!src || !dst || n < 1 || (slots != 8 && slots != 18) || nset < 1) return LPM_ERR_ARG;
    return ret(launch_pack<float>(src, dst, n, slots, nset, S(stream)));
}

int lpm_pack_coef_f64(const double* src, double* dst, int64_t n, int32_t slots, int32_t nset, void* stream)
{
    if (!src || !dst || n < 1 || (slots != 8 && slots != 18) || nset < 1) return LPM_ERR_ARG;
    return ret(launch_pack<double>(src, dst, n, slots, nset, S(stream)));
}

int64_t lpm_kmv_scratch_bytes(const lpm_lattice* lat, int32_t precision, int32_t nsys)
{
    Lattice L;
    if (to_lattice(lat, L) || nsys < 1) return LPM_ERR_ARG;
    const size_t es = precision == LPM_F32 ? 4 : 8;
    // FP32: room for the two pair-layout copies of the pair-packed operator (at most nsys pairs of 6 values)
    const size_t per = precision == LPM_F32 ? 12 : 4;
    return (int64_t)((size_t)nsys * L.N * per * es + 256);
}

int lpm_kmv_sc_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* out, void* scratch, size_t scratch_bytes, void* stream)
{
    return kmv_impl<double>(3, lat, u, Kn, Tv, coef_layout, batch, out, scratch, scratch_bytes, stream);
}
int lpm_kmv_sc_f32(const lpm_lattice* lat, const float* u, const float* Kn, const float* Tv, int32_t coef_layout,
                   const lpm_batch* batch, float* out, void* scratch, size_t scratch_bytes, void* stream)
{
    return kmv_impl<float>(3, lat, u, Kn, Tv, coef_layout, batch, out, scratch, scratch_bytes, stream);
}
int lpm_kmv_sq_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* out, void* scratch, size_t scratch_bytes, void* stream)
{
    return kmv_impl<double>(2, lat, u, Kn, Tv, coef_layout, batch, out, scratch, scratch_bytes, stream);
}
int lpm_kmv_sq_f32(const lpm_lattice* lat, const float* u, const float* Kn, const float* Tv, int32_t coef_layout,
                   const lpm_batch* batch, float* out, void* scratch, size_t scratch_bytes, void* stream)
{
    return kmv_impl<float>(2, lat, u, Kn, Tv, coef_layout, batch, out, scratch, scratch_bytes, stream);
}

int lpm_block_jacobi_f64(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                         int32_t nset, double* Minv, double* D_or_null, void* stream)
{
    Lattice L;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_layout(coef_layout, L, cl))) return rc;
    if (!Kn || !Tv || !Minv || nset < 1) return LPM_ERR_ARG;
    return ret(launch_block_jacobi<double>(L, Kn, Tv, cl, nset, Minv, D_or_null, S(stream)));
}

int lpm_block_jacobi_f32(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                         int32_t nset, float* Minv, double* D_or_null, void* stream)
{
    Lattice L;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_layout(coef_layout, L, cl))) return rc;
    if (!Kn || !Tv || !Minv || nset < 1) return LPM_ERR_ARG;
    return ret(launch_block_jacobi<float>(L, Kn, Tv, cl, nset, Minv, D_or_null, S(stream)));
}

int64_t lpm_cg_workspace_bytes(const lpm_lattice* lat, const lpm_batch* batch, int32_t precision, int32_t precond)
{
    Lattice L;
    Batch bt;
    if (to_lattice(lat, L) || to_batch(batch, bt)) return LPM_ERR_ARG;
    return (int64_t)cg_workspace_bytes(L, bt, precision, precond) + 256;
}

int lpm_cg_persistent_fits(const lpm_lattice* lat, const lpm_batch* batch, int32_t precision)
{
    Lattice L;
    Batch bt;
    if (to_lattice(lat, L) || to_batch(batch, bt)) return LPM_ERR_ARG;
    if (precision != LPM_F64 && precision != LPM_F32) return LPM_ERR_ARG;
    return persist_auto(L, bt, precision == LPM_F64 ? 8 : 4) ? 1 : 0;
}

int lpm_cg_batched_f64(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                       const lpm_batch* batch, const double* Minv, const uint8_t* mask, const double* b, double* x,
                       int32_t x_is_zero, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                       int32_t* iters, double* relres, int32_t* status, void* stream)
{
    return cg_impl<double>(lat, Kn, Tv, coef_layout, batch, Minv, mask, b, x, x_is_zero, opts, workspace,
                           workspace_bytes, iters, relres, status, stream);
}

int lpm_cg_batched_f32(const lpm_lattice* lat, const float* Kn, const float* Tv, int32_t coef_layout,
                       const lpm_batch* batch, const float* Minv, const uint8_t* mask, const float* b, float* x,
                       int32_t x_is_zero, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                       int32_t* iters, double* relres, int32_t* status, void* stream)
{
    return cg_impl<float>(lat, Kn, Tv, coef_layout, batch, Minv, mask, b, x, x_is_zero, opts, workspace,
                          workspace_bytes, iters, relres, status, stream);
}

int64_t lpm_ir_workspace_bytes(const lpm_lattice* lat, const lpm_batch* batch, int32_t precond)
{
    Lattice L;
    Batch bt;
    if (to_lattice(lat, L) || to_batch(batch, bt)) return LPM_ERR_ARG;
    return (int64_t)ir_workspace_bytes(L, bt, precond) + 256;
}

int lpm_ir_batched(const lpm_lattice* lat, const double* Kn64, const double* Tv64, int32_t coef_layout64,
                   const float* Kn32, const float* Tv32, const float* Minv32, const lpm_batch* batch,
                   const uint8_t* mask, const double* b, double* x, const lpm_ir_opts* opts, void* workspace,
                   size_t workspace_bytes, int32_t* iters, double* relres, int32_t* status, int32_t* outer_steps,
                   void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl64, cl32;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(coef_layout64, L, cl64)) ||
        (rc = to_layout(LPM_LAYOUT_SOA, L, cl32)))
        return rc;
    if (!Kn64 || !Tv64 || !Kn32 || !Tv32 || !b || !x || !opts || !workspace || !iters || !relres || !status)
        return LPM_ERR_ARG;
    if (!(opts->tol >= 0.0) || !(opts->inner_tol > 0.0)) return LPM_ERR_ARG;
    return ir_solve(L, Kn64, Tv64, cl64, Kn32, Tv32, cl32, Minv32, bt, mask, b, x, *opts, workspace,
                    workspace_bytes, iters, relres, status, outer_steps, S(stream));
}

int lpm_ir_amg(const lpm_lattice* lat, const double* Kn64, const double* Tv64, int32_t coef_layout64, lpm_amg* amg,
               const lpm_batch* batch, const uint8_t* mask, const double* b, double* x, const lpm_ir_opts* opts,
               void* workspace, size_t workspace_bytes, int32_t* iters, double* relres, int32_t* status,
               int32_t* outer_steps, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl64, cl32;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(coef_layout64, L, cl64)) ||
        (rc = to_layout(LPM_LAYOUT_SOA, L, cl32)))
        return rc;
    if (!amg || !Kn64 || !Tv64 || !b || !x || !opts || !workspace || !iters || !relres || !status) return LPM_ERR_ARG;
    if (!(opts->tol >= 0.0) || !(opts->inner_tol > 0.0)) return LPM_ERR_ARG;
    if (!amg_matches(amg, L, bt)) return LPM_ERR_ARG;
    return ir_solve(L, Kn64, Tv64, cl64, nullptr, nullptr, cl32, nullptr, bt, mask, b, x, *opts, workspace,
                    workspace_bytes, iters, relres, status, outer_steps, S(stream), amg);
}

int64_t lpm_grad_scratch_bytes(const lpm_lattice* lat, int32_t nsys)
{
    Lattice L;
    if (to_lattice(lat, L) || nsys < 1) return LPM_ERR_ARG;
    return (int64_t)(2 * (size_t)nsys * L.N * 4 * sizeof(double) + 256);
}

static int grad_impl(int dim, const lpm_lattice* lat, const double* u, const double* lam, const double* Kn,
                     const double* Tv, int32_t layout, const lpm_batch* batch, double* gKn, double* gTv,
                     int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc) return rc;
    if (L.dim != dim) return LPM_ERR_UNSUPPORTED;
    if ((rc = to_batch(batch, bt)) || (rc = to_layout(layout, L, cl))) return rc;
    if (!u || !lam || !Kn || !Tv || !gKn || !gTv) return LPM_ERR_ARG;
    double* st = nullptr;
    if (dim == 3) {
        st = aligned<double>(scratch, scratch_bytes, 2 * (size_t)bt.nsys * L.N * 4 * sizeof(double), rc);
        if (rc) return rc;
    }
    return ret(launch_grad(L, u, lam, Kn, Tv, cl, bt, gKn, gTv, st, accumulate, S(stream)));
}

int lpm_bond_grad_sc(const lpm_lattice* lat, const double* u, const double* lam, const double* Kn, const double* Tv,
                     int32_t coef_layout, const lpm_batch* batch, double* gKn, double* gTv, int32_t accumulate,
                     void* scratch, size_t scratch_bytes, void* stream)
{
    return grad_impl(3, lat, u, lam, Kn, Tv, coef_layout, batch, gKn, gTv, accumulate, scratch, scratch_bytes,
                     stream);
}

int lpm_bond_grad_sq(const lpm_lattice* lat, const double* u, const double* lam, const double* Kn, const double* Tv,
                     int32_t coef_layout, const lpm_batch* batch, double* gKn, double* gTv, int32_t accumulate,
                     void* scratch, size_t scratch_bytes, void* stream)
{
    return grad_impl(2, lat, u, lam, Kn, Tv, coef_layout, batch, gKn, gTv, accumulate, scratch, scratch_bytes,
                     stream);
}

int lpm_stress_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, const double* l0, double V, double* sig, void* scratch,
                   size_t scratch_bytes, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(coef_layout, L, cl))) return rc;
    if (!u || !Kn || !Tv || !l0 || !sig || !(V > 0.0)) return LPM_ERR_ARG;
    double* st = aligned<double>(scratch, scratch_bytes, (size_t)bt.nsys * L.N * 4 * sizeof(double), rc);
    if (rc) return rc;
    return ret(launch_stress(L, u, Kn, Tv, cl, bt, l0, V, sig, st, S(stream)));
}

int lpm_energy_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* w, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(coef_layout, L, cl))) return rc;
    if (!u || !Kn || !Tv || !w) return LPM_ERR_ARG;
    return ret(launch_energy(L, u, Kn, Tv, cl, bt, w, S(stream)));
}

static int vjp_impl(int which, const lpm_lattice* lat, const double* u, const double* G, const double* Kn,
                    const double* Tv, int32_t layout, const lpm_batch* batch, const double* l0, double V, double* du,
                    double* gKn, double* gTv, int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream)
{
    Lattice L;
    Batch bt;
    CoefLayout cl;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt)) || (rc = to_layout(layout, L, cl))) return rc;
    if (!u || !G || !Kn || !Tv || !du || !gKn || !gTv) return LPM_ERR_ARG;
    if (which == 1 && (!l0 || !(V > 0.0))) return LPM_ERR_ARG;
    double* st = aligned<double>(scratch, scratch_bytes, 2 * (size_t)bt.nsys * L.N * 4 * sizeof(double), rc);
    if (rc) return rc;
    return ret(launch_post_vjp(L, which, u, G, Kn, Tv, cl, bt, l0, V, du, gKn, gTv, st, accumulate, S(stream)));
}

int lpm_energy_vjp_f64(const lpm_lattice* lat, const double* u, const double* G, const double* Kn, const double* Tv,
                       int32_t coef_layout, const lpm_batch* batch, double* du, double* gKn, double* gTv,
                       int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream)
{
    return vjp_impl(0, lat, u, G, Kn, Tv, coef_layout, batch, nullptr, 1.0, du, gKn, gTv, accumulate, scratch,
                    scratch_bytes, stream);
}

int lpm_stress_vjp_f64(const lpm_lattice* lat, const double* u, const double* Gsig, const double* Kn,
                       const double* Tv, int32_t coef_layout, const lpm_batch* batch, const double* l0, double V,
                       double* du, double* gKn, double* gTv, int32_t accumulate, void* scratch, size_t scratch_bytes,
                       void* stream)
{
    return vjp_impl(1, lat, u, Gsig, Kn, Tv, coef_layout, batch, l0, V, du, gKn, gTv, accumulate, scratch,
                    scratch_bytes, stream);
}

int lpm_kmv_vjp_f64(const lpm_lattice* lat, const double* u, const double* G, const double* Kn, const double* Tv,
                    int32_t coef_layout, const lpm_batch* batch, double* du, double* gKn, double* gTv,
                    int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream)
{
    if (lat && lat->dim != 3) return LPM_ERR_UNSUPPORTED;
    return vjp_impl(2, lat, u, G, Kn, Tv, coef_layout, batch, nullptr, 1.0, du, gKn, gTv, accumulate, scratch,
                    scratch_bytes, stream);
}

int lpm_autotune_kmv(const lpm_lattice* lat, const lpm_batch* batch, const float* Kn, const float* Tv, void* scratch,
                     size_t scratch_bytes, int32_t* zchunk_out, int32_t* variant_out, void* stream)
{
    Lattice L;
    Batch bt;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt))) return rc;
    if (!Kn || !Tv || !zchunk_out) return LPM_ERR_ARG;
    if (L.dim != 3 || L.nbr || !pair_supported(L.nx) || !tma_aligned(Kn, Tv, Kn)) return LPM_ERR_UNSUPPORTED;
    const int npp = (bt.rhs_per_set + 1) / 2, nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    const size_t nvp = (size_t)nset * npp * L.N * 6;
    float* up = aligned<float>(scratch, scratch_bytes, 2 * nvp * sizeof(float), rc);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    cudaError_t e = cudaMemsetAsync(up, 0, nvp * sizeof(float), st);
    PairArgs a{};
    a.nx = L.nx;
    a.ny = L.ny;
    a.nz = L.nz;
    a.N = L.N;
    a.nsys = bt.nsys;
    a.rhs_per_set = bt.rhs_per_set;
    a.npp = npp;
    a.npair = nset * npp;
    a.u = up;
    a.Kn = Kn;
    a.Tv = Tv;
    a.out = up + nvp;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int best = pair_zchunk_heuristic(L.nx, L.ny, L.nz, a.npair), best_var = kPairDefaultVariant;
    float best_ms = 0.f;
    bool have = false;
    for (int var = 0; var < 2; ++var) {
        for (int nzc = 1; e == cudaSuccess && nzc <= pair_zchunk_max_chunks(L.nz); ++nzc) {
            const int zc = (L.nz + nzc - 1) / nzc;
            if (nzc > 1 && (L.nz + zc - 1) / zc != nzc) continue;  // same chunking as a smaller count
            a.zchunk = zc;
            a.variant = var;
            e = launch_sc_pair(a, false, st);  // warm-up
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventRecord(e0, st);
            for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch_sc_pair(a, false, st);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && (!have || ms < best_ms)) {
                best_ms = ms;
                best = zc;
                best_var = var;
                have = true;
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return ret(e);
    pair_zchunk_record(L.nx, L.ny, L.nz, a.npair, best, best_var);
    *zchunk_out = best;
    if (variant_out) *variant_out = best_var;
    return LPM_OK;
}

int lpm_tune_kmv_set(const lpm_lattice* lat, const lpm_batch* batch, int32_t zchunk, int32_t variant)
{
    Lattice L;
    Batch bt;
    int rc = to_lattice(lat, L);
    if (rc || (rc = to_batch(batch, bt))) return rc;
    if (L.dim != 3 || zchunk < 1 || zchunk > L.nz || (L.nz + zchunk - 1) / zchunk > pair_zchunk_max_chunks(L.nz) ||
        (variant != 0 && variant != 1))
        return LPM_ERR_ARG;
    const int npp = (bt.rhs_per_set + 1) / 2, nset = (bt.nsys + bt.rhs_per_set - 1) / bt.rhs_per_set;
    pair_zchunk_record(L.nx, L.ny, L.nz, nset * npp, zchunk, variant);
    return LPM_OK;
}

int lpm_solid_nbr(int32_t dim, int32_t nx, int32_t ny, int32_t nz, int32_t nspec, const uint8_t* solid, int32_t* nbr,
                  void* stream)
{
    if ((dim != 2 && dim != 3) || nx < 1 || ny < 1 || nz < 1 || (dim == 2 && nz != 1) || nspec < 1 || nspec > 65535 ||
        !solid || !nbr || (int64_t)nx * ny * nz > INT32_MAX)
        return LPM_ERR_ARG;
    return ret(launch_solid_nbr(dim, nx, ny, nz, nspec, solid, nbr, S(stream)));
}

int lpm_build_nbr(int32_t dim, int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t* site_of,
                  const int64_t* sites, int64_t* nbr, void* stream)
{
    if ((dim != 2 && dim != 3) || nx < 1 || ny < 1 || nz < 1 || n < 0 || (dim == 2 && nz != 1)) return LPM_ERR_ARG;
    if (n > 0 && (!site_of || !sites || !nbr)) return LPM_ERR_ARG;
    return ret(launch_build_nbr(dim, nx, ny, nz, n, site_of, sites, nbr, S(stream)));
}

}  // extern "C"
