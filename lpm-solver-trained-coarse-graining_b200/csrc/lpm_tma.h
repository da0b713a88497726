// TMA-fed fused SC operator: launch arguments and configuration helpers.
#pragma once
#include <cuda.h>

#include "lpm_fused.h"

namespace lpm {

template <typename T>
struct TmaArgs {
    int nx, ny, nz;
    int64_t N;
    int nsys, rhs_per_set, nmask;
    int nr;      // systems per CTA
    int ngrp;    // CTA groups per coefficient set = ceil(rhs_per_set / nr)
    int set0;    // first coefficient set of this launch (grid.y chunking)
    int zchunk;  // z planes per CTA
    const T* u;  // (nsys, N, 3)
    const T* Kn; // (nset, 18, N)
    const T* Tv;
    T* out;      // (nsys, N, 3)
    const uint8_t* mask;  // epilogue: per-DOF free mask (nmask, N, 3) or nullptr
    const int* act;       // optional activity flags (inactive systems are skipped)
    double* part;         // epilogue: per-system partials (nsys, nblk) or nullptr
    unsigned* cnt;        // epilogue: per-system last-block counters
    FcgScalars scv;       // epilogue: alpha step of the CG engine when has_sc
    int has_sc;
    int it;
    int* err;             // set to 1 if an mbarrier wait expired
    unsigned wait_polls;  // poll bound of the data waits (set by the launcher from tma_wait_polls())
};

// Tiled 4D tensor map over FP32 (elem_bytes 4) or FP64 data, no swizzle, zero fill out of bounds; false when the
// driver entry point is missing or the encoding is rejected.
// Poll bound of the TMA operators' data waits (process-wide; default ptx::kWaitLimit).  Setting it returns the
// previous bound; 0 makes every data wait expire at once, so the kernels take their abort path (record the error,
// let the copies they issued land with the full bound, stop computing).
unsigned tma_wait_polls();
unsigned tma_set_wait_polls(unsigned polls);

bool make_tensor_map4(CUtensorMap* m, int elem_bytes, const void* base, const uint64_t dims[4],
                      const uint64_t strides_bytes[3], const uint32_t box[4]);
bool tma_supported(int nx, int elem_bytes);
bool tma_aligned(const void* a, const void* b, const void* c);  // 16-byte aligned global bases
int tma_group_size(int rhs_per_set, int elem_bytes);
int tma_tile_rows(int elem_bytes);
int tma_zchunk(int nx, int ny, int nz, int nset, int ngrp, int elem_bytes);
int tma_dot_blocks_max(int nx, int ny, int nz, int elem_bytes);

template <typename T>
cudaError_t launch_sc_tma(const TmaArgs<T>& a, bool epi, cudaStream_t st);

// Pair-packed FP32 operator (kmv_pair.cu): vectors in the pair layout (npair, N, 3, 2), pair = set * npp + j / 2,
// lane = j % 2 for system j of a set; unmasked output; epilogue as above.  Its FP64 instantiation (one system per
// lane group) takes natural-layout vectors: launch_sc_pair64 below.
struct PairArgs {
    int nx, ny, nz;
    int64_t N;
    int nsys, rhs_per_set;
    int npp;     // pairs per coefficient set = ceil(rhs_per_set / 2)
    int npair;   // pairs in the batch = nset * npp
    int set0;    // first coefficient set of this launch (grid.y chunking)
    int zchunk;  // z planes per CTA
    int variant; // 0: staged (Tv, Kn through shared memory, one CTA per SM); 1: lean (two CTAs per SM)
    const float* u;   // pair layout
    const float* Kn;  // (nset, 18, N)
    const float* Tv;
    float* out;       // pair layout
    const int* act;
    double* part;
    unsigned* cnt;
    FcgScalars scv;
    int has_sc;
    int it;
    int* err;
    unsigned wait_polls;  // poll bound of the data waits (set by the launcher from tma_wait_polls())
    // AMG smoother epilogues (PM_RESID, PM_SMOOTH, PM_SMOOTH_DOT)
    const float* rhs;  // pair layout: the right-hand side of the smoothing step
    const float* Ms;   // (nset, 9, N) block-Jacobi inverse
    const int* fbox;   // (nsys, 6) free box of every system: lo x, y, z, hi x, y, z (inclusive)
    const float* fw;   // (nsys) smoother weight omega / rho
};

// Epilogues of the pair operator.  f = K u per site and lane; m = 1 inside the lane's free box, else 0.
enum PairMode {
    PM_NONE = 0,       // out = f
    PM_DOT = 1,        // out = f; u.f per system, the last block runs the CG alpha step
    PM_RESID = 2,      // out = m (rhs - f)
    PM_SMOOTH = 3,     // out = u + w m M (rhs - f)            (damped block-Jacobi sweep)
    PM_SMOOTH_DOT = 4  // as PM_SMOOTH; rhs.out per system, the last block runs the PCG beta step
};

bool pair_supported(int nx);
constexpr int kPairDefaultVariant = 0;
int pair_zchunk(int nx, int ny, int nz, int npair);            // autotuned value if recorded, else heuristic
int pair_variant(int nx, int ny, int nz, int npair);           // autotuned variant if recorded, else the default
int pair_zchunk_heuristic(int nx, int ny, int nz, int npair);
void pair_zchunk_record(int nx, int ny, int nz, int npair, int zchunk, int variant);
int pair_zchunk_max_chunks(int nz);                               // z chunks allowed (>= 8 planes each)
int pair_dot_blocks_max(int nx, int ny, int nz);
cudaError_t launch_sc_pair(const PairArgs& a, bool epi, cudaStream_t st);
cudaError_t launch_sc_pair_mode(const PairArgs& a, int mode, cudaStream_t st);
// FP64 instantiation (lean variant, one system per lane group): u and out natural-layout (nsys, N, 3) FP64 arrays and
// Kn / Tv packed FP64 coefficients, all passed through PairArgs' float pointers; npp = rhs_per_set, npair = nset *
// npp.  epi: PM_DOT (u.out per system into part / cnt, and the CG alpha step when has_sc).
bool pair64_supported(int nx);
cudaError_t launch_sc_pair64(const PairArgs& a, bool epi, cudaStream_t st);
// Arguments of the FP64 operator for a batch (no epilogue fields set).
PairArgs pair64_args(int nx, int ny, int nz, int64_t N, int nsys, int rps, const double* u, const double* Kn,
                     const double* Tv, double* out);
// Shared-memory opt-in of every pair-operator kernel on the current device (call before capturing launches).
cudaError_t pair_prepare();
// (nsys, N, 3) FP32 -> pair layout (dummy lanes written as zero) and back (real systems only); npair <= 65535.
cudaError_t pair_pack(const float* x, float* xp, int64_t N, int nsys, int rps, cudaStream_t st);
cudaError_t pair_unpack(const float* xp, float* x, int64_t N, int nsys, int rps, cudaStream_t st);

// Fills the configuration fields of a TmaArgs for a batch (nr, ngrp, zchunk).
template <typename T>
inline void tma_configure(TmaArgs<T>& a)
{
    const int es = (int)sizeof(T);
    a.nr = tma_group_size(a.rhs_per_set, es);
    a.ngrp = (a.rhs_per_set + a.nr - 1) / a.nr;
    a.zchunk = tma_zchunk(a.nx, a.ny, a.nz, (a.nsys + a.rhs_per_set - 1) / a.rhs_per_set, a.ngrp, es);
}

}  // namespace lpm
