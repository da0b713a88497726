// Internal launcher declarations of the LPM CUDA library (host side; not part of the C ABI).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "lpm_common.cuh"

namespace lpm {

// Lattice description shared by all launchers.  For structured boxes nbr == nullptr and neighbours are implicit
// (site id (z*ny + y)*nx + x); otherwise nbr is an (N, NN) int32 table with -1 for a missing bond.
struct Lattice {
    int dim;  // 2 (square, 8 slots) or 3 (simple cubic, 18 slots)
    int nx, ny, nz;
    int64_t N;
    const int32_t* nbr;
};

inline int slots_of(const Lattice& L) { return L.dim == 3 ? 18 : 8; }

// Masked-CG epilogue options of the operator launch.
// When dot_part is set, the launch reduces in . out per system deterministically: per-block partials go to
// dot_part (nsys, kmv_dot_blocks(L)), the last block of each system sums them in fixed order into dot_final[s] and
// re-arms counter[s] (which must start at 0).
struct MvEpilogue {
    const uint8_t* mask;  // per-DOF free mask (nmask, N, d) or nullptr (no masking)
    double* dot_part;
    double* dot_final;
    unsigned* counter;
    const int* act;       // optional per-system activity flags: inactive systems are skipped (output untouched)
    // Optional fused CG p-update (full 2D boxes through the 2D tile kernels; the launcher reports
    // cudaErrorNotSupported elsewhere): the operator's input is p' = z + beta[s] p, formed while staging the tile, with p and p' in the two
    // buffers p0 / p1 (the previous p in p0 when pk[s] is even), and p' of the tile's own sites is stored.  The
    // input pointer u of the launch is then unused.
    const void* pz = nullptr;      // z (r for plain CG), (nsys, N, d)
    void* p0 = nullptr;            // p buffers, (nsys, N, d) each
    void* p1 = nullptr;
    const double* beta = nullptr;  // beta of the step that forms p'
    const int* pk = nullptr;       // completed iterations per system (the buffer parity)
};

// out = K u for every system of the batch.  scratch: (nsys, N, 4) values of type T.
template <typename T>
cudaError_t launch_kmv(const Lattice& L, const T* u, const T* Kn, const T* Tv, const CoefLayout& cl, const Batch& bt,
                       T* out, T* scratch, const MvEpilogue* ep, cudaStream_t st);

// Pass 1 only: per-particle shell sums (S0, S1, TS0, TS1) of every system into st (nsys, N, 4).
template <typename T>
cudaError_t launch_kmv_sums(const Lattice& L, const T* u, const T* Tv, const CoefLayout& cl, const Batch& bt, T* st,
                            cudaStream_t stream);

// Number of dot partials per system that launch_kmv writes when ep->dot_part is set.
int kmv_dot_blocks(const Lattice& L);

// Preconditioner: inverse diagonal blocks (nset, N, d, d) of K for each coefficient set (values in T, built in FP64).
template <typename T>
cudaError_t launch_block_jacobi(const Lattice& L, const double* Kn, const double* Tv, const CoefLayout& cl, int nset,
                                T* Minv, double* D_out, cudaStream_t st);

// Pack (nset, N, NN) FP64 coefficients into the SoA layout (nset, NN, N) of type T.
template <typename T>
cudaError_t launch_pack(const double* src, T* dst, int64_t N, int NN, int nset, cudaStream_t st);

// Per-slot gradient of sum_s lam_s . K u_s over the systems of each coefficient set (sign: +).
cudaError_t launch_grad(const Lattice& L, const double* u, const double* lam, const double* Kn, const double* Tv,
                        const CoefLayout& cl, const Batch& bt, double* gKn, double* gTv, double* scratch,
                        int accumulate, cudaStream_t st);

// Post-processing: particle stress (nsys, N, 3 or 6) and particle energy (nsys, N).
cudaError_t launch_stress(const Lattice& L, const double* u, const double* Kn, const double* Tv, const CoefLayout& cl,
                          const Batch& bt, const double* l0, double V, double* sig, double* scratch, cudaStream_t st);
cudaError_t launch_energy(const Lattice& L, const double* u, const double* Kn, const double* Tv, const CoefLayout& cl,
                          const Batch& bt, double* w, cudaStream_t st);

// VJPs of the particle energy (which = 0, G (nsys, N)) or stress (which = 1, G (nsys, N, 6 or 3)): du (nsys, N, d)
// and parameter gradients (nset, N, NN) summed over the systems of each set.  scratch: 2 * nsys * N * 4 doubles.
cudaError_t launch_post_vjp(const Lattice& L, int which, const double* u, const double* G, const double* Kn,
                            const double* Tv, const CoefLayout& cl, const Batch& bt, const double* l0, double V,
                            double* du, double* gK, double* gT, double* scratch, int acc, cudaStream_t st);

// Per-specimen bond tables (nspec, nx*ny*nz, NN) int32 of a full box with per-specimen solid masks (nspec, n) uint8.
cudaError_t launch_solid_nbr(int dim, int nx, int ny, int nz, int nspec, const uint8_t* solid, int32_t* nbr,
                             cudaStream_t st);

// Neighbour table (n, NN) int64 of a masked box, same values as the reference's LatticeGeom.nbr.
cudaError_t launch_build_nbr(int dim, int nx, int ny, int nz, int64_t n, const int64_t* site_of, const int64_t* sites,
                             int64_t* nbr, cudaStream_t st);

}  // namespace lpm
