// TMA-fed fused SC operator: launch arguments and configuration helpers.
#pragma once
#include "lpm_fused.h"

namespace lpm {

template <typename T>
struct TmaArgs {
    int nx, ny, nz;
    int64_t N;
    int nsys, rhs_per_set, nmask;
    int nr;      // systems per CTA
    int ngrp;    // CTA groups per coefficient set = ceil(rhs_per_set / nr)
    int grp0;    // first group of this launch (grid.y chunking)
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
};

bool tma_supported(int nx, int elem_bytes);
bool tma_aligned(const void* a, const void* b, const void* c);  // 16-byte aligned global bases
int tma_group_size(int rhs_per_set, int elem_bytes);
int tma_tile_rows(int elem_bytes);
int tma_zchunk(int nx, int ny, int nz, int nset, int ngrp, int elem_bytes);
int tma_dot_blocks_max(int nx, int ny, int nz, int elem_bytes);

template <typename T>
cudaError_t launch_sc_tma(const TmaArgs<T>& a, bool epi, cudaStream_t st);

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
