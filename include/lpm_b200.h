/*
 * lpm_b200.h -- C ABI of the B200 LPM linear-solve library (liblpm_b200.so).
 *
 * Matrix-free K.u of the linearised lattice particle model on the square (2D, 8 slots, 2 DOF) and simple-cubic (3D,
 * 18 slots, 3 DOF) lattices, batched CG / block-Jacobi PCG, FP32-inner / FP64-refinement solves, per-bond adjoint
 * gradients and stress / energy post-processing.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer owned by the caller (e.g. the data_ptr() of a torch tensor).  No entry
 *    point allocates device memory; scratch and workspace buffers are passed in, sized by the *_bytes queries.
 *  - Functions return 0 on success, a negative LPM_ERR_* code for a bad argument, or a positive cudaError_t value.
 *  - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default stream).  Solver entry points synchronise
 *    the stream every `poll` iterations to read one convergence counter; all other entry points are asynchronous.
 *  - No global mutable state: calls on distinct streams with distinct buffers are thread-safe.
 *  - Slot order, bond directions and particle numbering are those of the reference (coarse3d/geom3d.py:16-65,
 *    coarse2d/lin2d.py:21-74): slots in reverse pairs (k, k^1), shell 0 = axial bonds, n_k = -o_k/|o_k|.
 *  - Batches: nsys systems (right-hand sides); system s uses coefficient set s / rhs_per_set and DOF mask s % nmask.
 *    Vectors are (nsys, n, d) contiguous; coefficient sets (nset, n, slots) in the reference layout
 *    (LPM_LAYOUT_REF) or (nset, slots, n) packed (LPM_LAYOUT_SOA); masks (nmask, n, d) uint8, 1 = free DOF.
 */
#ifndef LPM_B200_H
#define LPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LPM_ABI_VERSION 4

/* return codes */
#define LPM_OK 0
#define LPM_ERR_ARG (-1)         /* invalid argument (null pointer, bad size, unsupported combination) */
#define LPM_ERR_WORKSPACE (-2)   /* workspace / scratch buffer too small */
#define LPM_ERR_UNSUPPORTED (-3) /* lattice or precision not supported by this entry point */
#define LPM_ERR_TIMEOUT (-5)     /* a bounded device-side wait expired (the kernel stopped and returned) */

/* per-system solver status */
#define LPM_STATUS_OK 0
#define LPM_STATUS_NOT_CONVERGED 1 /* maxit reached (mirrors lin3d._pcg returning maxit, solver2d's iters = -1) */
#define LPM_STATUS_BREAKDOWN 2     /* p.Ap < 0 or a non-finite scalar (mirrors torch_lpm's FloatingPointError) */

/* CG engines (lpm_cg_opts.engine, lpm_ir_opts.engine) */
#define LPM_ENGINE_AUTO 0       /* persistent where lpm_cg_persistent_fits says so and no timing is asked, else launched */
#define LPM_ENGINE_LAUNCHED 1   /* one launch per step; iteration blocks replayed as CUDA graphs, host polls */
#define LPM_ENGINE_PERSISTENT 2 /* one cooperative launch runs the whole solve (small batches) */

/* precisions and coefficient layouts */
#define LPM_F64 0
#define LPM_F32 1
#define LPM_LAYOUT_REF 0 /* (nset, n, slots): the reference's Kn / Tv arrays */
#define LPM_LAYOUT_SOA 1 /* (nset, slots, n): packed by lpm_pack_coef_* */

typedef struct lpm_lattice {
    int32_t dim;        /* 2: square lattice, 3: simple cubic */
    int32_t nx, ny, nz; /* box size in sites (nz = 1 in 2D) */
    int64_t n;          /* number of particles (= nx*ny*nz for a full box) */
    const int32_t* nbr; /* NULL: full box, implicit neighbours.  Else (n, slots) int32 table, -1 = no bond. */
} lpm_lattice;

typedef struct lpm_batch {
    int32_t nsys;        /* systems (right-hand sides) */
    int32_t rhs_per_set; /* consecutive systems sharing one coefficient set */
    int32_t nmask;       /* number of DOF masks; system s uses mask s % nmask */
    int32_t reserved;
} lpm_batch;

typedef struct lpm_cg_opts {
    double tol;       /* stop a system when |r| <= tol |b| */
    int32_t maxit;    /* iteration limit */
    int32_t check;    /* convergence test every `check` iterations (1 = lin3d._pcg, 10 = torch_lpm3d.SCT.pcg) */
    int32_t poll;     /* host reads the converged count every `poll` iterations */
    int32_t precheck; /* 1: test the initial residual before iterating (cg2plain.cg_mf / solver2d.pcg_mf) */
    double* prof;     /* optional HOST array of 4: K.u ms / launches, and the same for full-batch launches */
    const double* tol_sys; /* optional DEVICE array (nsys): per-system tolerance used instead of tol */
    int32_t engine;   /* LPM_ENGINE_*: 0 = auto */
    int32_t reserved;
} lpm_cg_opts;

typedef struct lpm_ir_opts {
    double tol;          /* FP64 true relative residual target |b - Kx| <= tol |b| */
    double inner_tol;    /* relative tolerance of each FP32 correction solve */
    int32_t maxit;       /* limit on the total inner iterations per system */
    int32_t max_outer;   /* limit on refinement steps */
    int32_t check;       /* inner convergence-test interval */
    int32_t poll;        /* inner host polling interval */
    double* prof;        /* optional HOST array of 4, as lpm_cg_opts.prof, for the FP32 inner solves */
    int32_t x_is_zero;   /* 1: x is zero on entry, so the first residual is b (no FP64 K x) */
    int32_t engine;      /* LPM_ENGINE_* of the FP32 inner solves: 0 = auto */
} lpm_ir_opts;

int lpm_abi_version(void);
const char* lpm_status_string(int code);
/* Diagnostics of the CUDA-graph cache behind the CG engines' iteration blocks: graphs captured so far, graphs held,
 * and evictions from the bounded (least-recently-used) cache, process-wide.  No counterpart in the reference (it has
 * no CUDA graphs). */
void lpm_graph_stats(int64_t* captures, int64_t* entries, int64_t* flushes);

/* ------------------------------------------------------------------------------------------------ coefficients */
/* Pack (nset, n, slots) FP64 coefficients into the (nset, slots, n) layout in FP32 or FP64.
 * Replaces the per-solve casts of timing/t2d/solver2d.py:570-575 (Sys.mf_arrays(fp32=True)). */
int lpm_pack_coef_f32(const double* src, float* dst, int64_t n, int32_t slots, int32_t nset, void* stream);
int lpm_pack_coef_f64(const double* src, double* dst, int64_t n, int32_t slots, int32_t nset, void* stream);

/* ----------------------------------------------------------------------------------------------------- K . u */
/* Scratch bytes of one lpm_kmv_* call for `nsys` systems. */
int64_t lpm_kmv_scratch_bytes(const lpm_lattice* lat, int32_t precision, int32_t nsys);

/* out = K u.  SC: code-force operator of coarse3d/lin3d.py:126-149 (k_apply) and coarse3d/torch_lpm3d.py:63-83
 * (SCT.apply, batched).  SQ: exact-Hessian operator of timing/t2d/solver2d.py:269-305 (_kmv). */
int lpm_kmv_sc_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* out, void* scratch, size_t scratch_bytes, void* stream);
int lpm_kmv_sc_f32(const lpm_lattice* lat, const float* u, const float* Kn, const float* Tv, int32_t coef_layout,
                   const lpm_batch* batch, float* out, void* scratch, size_t scratch_bytes, void* stream);
int lpm_kmv_sq_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* out, void* scratch, size_t scratch_bytes, void* stream);
int lpm_kmv_sq_f32(const lpm_lattice* lat, const float* u, const float* Kn, const float* Tv, int32_t coef_layout,
                   const lpm_batch* batch, float* out, void* scratch, size_t scratch_bytes, void* stream);

/* Size of the device array behind lpm_kmv_f64_static: 32 MiB on every GPU that loads the library, held until exit. */
#define LPM_KMV_STATIC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* FP64 out = K u, the same operator as lpm_kmv_sc_f64 (lat->dim == 3) or lpm_kmv_sq_f64 (lat->dim == 2) and equal to
 * it within rounding (this entry always runs the two-pass kernels; full SC boxes in the packed layout go through the
 * single-pass TMA operator there), but with no scratch
 * argument and no device allocation: for callers that cannot allocate device memory or pass a buffer (an FFI host
 * that only forwards device pointers it was given, a fixed memory budget, a path where a cudaMalloc would stall).
 * No counterpart in the reference.  Limit: 4 * nsys * n doubles must fit LPM_KMV_STATIC_SCRATCH_BYTES (nsys * n <=
 * 1,048,576, e.g. nine systems of a 48^3 box), else LPM_ERR_WORKSPACE.  The first call on a device looks up the
 * array's device address with that device current, so make it before any stream capture; the cached address does
 * not survive a cudaDeviceReset of that device.  Every call on a device
 * shares the array: calls whose work overlaps on the GPU race and must be serialised by the caller. */
int lpm_kmv_f64_static(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv,
                       int32_t coef_layout, const lpm_batch* batch, double* out, void* stream);

/* --------------------------------------------------------------------------------------------- preconditioner */
/* Diagonal blocks D (nset, n, d, d) of K (optional output, FP64) and their inverses Minv (nset, n, d, d).
 * SC: coarse3d/lin3d.py:239-301 (k_block_diag, k_block_jacobi), coarse3d/torch_lpm3d.py:22-33,94-106 (inv3,
 * block_diag, precond).  SQ: timing/t2d/solver2d.py:308-346 (_diag_inv).  Fixed particles are handled by the DOF mask
 * when the preconditioner is applied (z = mask (Minv r)), so Minv itself is not masked. */
int lpm_block_jacobi_f64(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                         int32_t nset, double* Minv, double* D_or_null, void* stream);
int lpm_block_jacobi_f32(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                         int32_t nset, float* Minv, double* D_or_null, void* stream);

/* ------------------------------------------------------------------------------------------------ batched CG */
/* Workspace bytes of lpm_cg_batched_* for this lattice and batch (precond: 1 if Minv will be passed). */
int64_t lpm_cg_workspace_bytes(const lpm_lattice* lat, const lpm_batch* batch, int32_t precision, int32_t precond);

/* Batched (P)CG on the free DOFs: K_ff x_f = b_f for every system, x updated in place (x must be zero on fixed DOFs;
 * x_is_zero = 1 skips the initial K x).  Replaces coarse3d/lin3d.py:464-532 (_pcg / solve_pcg),
 * timing/t3d/cgplain.py:11-55 (cg3), timing/t2d/cg2plain.py:11-49 (cg_mf), timing/t2d/solver2d.py:349-421
 * (pcg_mf) and coarse3d/torch_lpm3d.py:109-140 (SCT.pcg).  Minv NULL = plain CG.  Full SC boxes with packed
 * (LPM_LAYOUT_SOA) coefficients run on the fused single-pass operator.  Outputs per system: iterations,
 * relative residual |r|/|b| at the last test, LPM_STATUS_*.  coef_layout applies to Kn/Tv. */
int lpm_cg_batched_f64(const lpm_lattice* lat, const double* Kn, const double* Tv, int32_t coef_layout,
                       const lpm_batch* batch, const double* Minv, const uint8_t* mask, const double* b, double* x,
                       int32_t x_is_zero, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                       int32_t* iters, double* relres, int32_t* status, void* stream);
int lpm_cg_batched_f32(const lpm_lattice* lat, const float* Kn, const float* Tv, int32_t coef_layout,
                       const lpm_batch* batch, const float* Minv, const uint8_t* mask, const float* b, float* x,
                       int32_t x_is_zero, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                       int32_t* iters, double* relres, int32_t* status, void* stream);

/* 1 if the automatic engine choice runs this batch in `precision` (LPM_F64 / LPM_F32) on the persistent engine:
 * square-lattice batches of at most 2^17 particle-systems (either precision) that fit on teams of co-resident
 * blocks (every system's particles on one team).  The persistent engine keeps the launched engine's algorithm, tests and
 * freezing (same iteration counts up to the rounding of its reductions) and runs one cooperative kernel per solve:
 * three team barriers per iteration, each wait bounded in time (LPM_ERR_TIMEOUT on expiry). */
int lpm_cg_persistent_fits(const lpm_lattice* lat, const lpm_batch* batch, int32_t precision);

/* Bound of one team-barrier wait of the persistent engine, in ns (process-wide, default 2e9); returns the previous
 * bound.  A wait that exceeds it records LPM_ERR_TIMEOUT, the kernel's blocks return and the solve reports that code.
 * 0 makes every wait that does not find its barrier passed at once expire: the way a test exercises the expiry path
 * without hanging or faulting a GPU.  No counterpart in the reference (it has no device-side waits). */
uint64_t lpm_set_wait_limit_ns(uint64_t ns);

/* Bound of the TMA-fed operators' data waits, in mbarrier polls (process-wide, default 4194304); returns the previous
 * bound.  An expired wait makes the kernel record the error, let the copies it issued land (with the default bound)
 * and stop computing; the CG engines then return LPM_ERR_TIMEOUT.  0 makes every data wait expire at once: the way a
 * test exercises the abort path without hanging or faulting a GPU.  No counterpart in the reference. */
uint32_t lpm_set_tma_wait_polls(uint32_t polls);

/* ------------------------------------------------------------------------------------- assembled matrices */
/* Workspace bytes of lpm_csr_pcg_f64 for an n x n matrix. */
int64_t lpm_csr_workspace_bytes(int64_t n);

/* K_ff x_f = b_f for an assembled sparse K (CSR: rowptr (n+1) int64, col int32, val FP64, device arrays) with the free
 * set as a per-row mask (uint8, 1 = free; NULL = all free), by Jacobi-preconditioned CG in FP64 from x = 0, stopping
 * when |r| <= tol |b| (tested every iteration).  x (n) receives the free part (zero on fixed rows); b is read on free
 * rows only.  Replaces the SuperLU factorisation and solve of coarse2d/lin2d.py:166-180 (solve_disp), called from
 * coarse2d/cg.py:64-76 for the 2D fine references.  opts: tol, maxit and poll are used (prof non-NULL turns off the
 * graph replay).  iters / relres / status: DEVICE arrays of one element. */
int lpm_csr_pcg_f64(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val, const uint8_t* mask,
                    const double* b, double* x, const lpm_cg_opts* opts, void* workspace, size_t workspace_bytes,
                    int32_t* iters, double* relres, int32_t* status, void* stream);

/* ------------------------------------------------------------------------------- mixed-precision refinement */
int64_t lpm_ir_workspace_bytes(const lpm_lattice* lat, const lpm_batch* batch, int32_t precond);

/* FP32 inner PCG + FP64 iterative refinement to |b - K x| <= tol |b| on the FP64 operator.
 * Kn64/Tv64: FP64 coefficients (coef_layout64); Kn32/Tv32: the same packed to FP32 SoA (lpm_pack_coef_f32);
 * Minv32: FP32 block-Jacobi inverse or NULL.  x (FP64) updated in place, zero on fixed DOFs on entry.
 * Each refinement step solves K d = r/|r| of system s by FP32 PCG to the relative tolerance
 * max(inner_tol, tol / (4 rel_s)), rel_s its FP64 relative residual (inexact refinement: the last step reduces only
 * what is left; a system's iterations never depend on the other systems of the batch).  Outputs: total inner iterations, final FP64 relative residual, status per system (device arrays);
 * outer_steps is a HOST pointer (may be NULL) that receives the number of refinement steps. */
int lpm_ir_batched(const lpm_lattice* lat, const double* Kn64, const double* Tv64, int32_t coef_layout64,
                   const float* Kn32, const float* Tv32, const float* Minv32, const lpm_batch* batch,
                   const uint8_t* mask, const double* b, double* x, const lpm_ir_opts* opts, void* workspace,
                   size_t workspace_bytes, int32_t* iters, double* relres, int32_t* status, int32_t* outer_steps,
                   void* stream);

/* ------------------------------------------------------------------------------------------------ gradients */
int64_t lpm_grad_scratch_bytes(const lpm_lattice* lat, int32_t nsys);

/* Per-slot derivatives of sum_s lam_s . K(Kn, Tv) u_s, summed over the systems of each coefficient set, written (or
 * added, accumulate = 1) to gKn, gTv (nset, n, slots) in the reference layout; zero on missing bonds.
 * SC (code-force operator): the autograd pass of coarse3d/torch_lpm3d.py:165-175 (LinSolve.backward) in closed form.
 * SQ (exact Hessian): the gradient of coarse2d/torch_lpm.py:173-191 (assemble) through 34-51 (SPDSolve.backward).
 * The adjoint solve's loss gradient is minus these values. */
int lpm_bond_grad_sc(const lpm_lattice* lat, const double* u, const double* lam, const double* Kn, const double* Tv,
                     int32_t coef_layout, const lpm_batch* batch, double* gKn, double* gTv, int32_t accumulate,
                     void* scratch, size_t scratch_bytes, void* stream);
int lpm_bond_grad_sq(const lpm_lattice* lat, const double* u, const double* lam, const double* Kn, const double* Tv,
                     int32_t coef_layout, const lpm_batch* batch, double* gKn, double* gTv, int32_t accumulate,
                     void* scratch, size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------------------------------ post-processing */
/* Particle stress with the opp-flag surface rule: SC (nsys, n, 6) xx yy zz yz xz xy (coarse3d/lin3d.py:170-210);
 * SQ (nsys, n, 3) xx yy xy (timing/t2d/solver2d.py:220-256).  l0: bond length per slot (slots,), V: particle volume.
 * scratch: lpm_kmv_scratch_bytes(lat, LPM_F64, nsys). */
int lpm_stress_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, const double* l0, double V, double* sig, void* scratch,
                   size_t scratch_bytes, void* stream);
/* Particle energy (nsys, n) (coarse3d/lin3d.py:213-236, coarse2d/lin2d.py:156-163). */
int lpm_energy_f64(const lpm_lattice* lat, const double* u, const double* Kn, const double* Tv, int32_t coef_layout,
                   const lpm_batch* batch, double* w, void* stream);

/* Vector-Jacobian products of the post-processing outputs, for differentiable solves (the autograd passes of
 * coarse3d/torch_lpm3d.py:85-92 and coarse2d/torch_lpm.py:246-258).  G: upstream gradient of the particle energy
 * (nsys, n) or of the stress (nsys, n, 6 | 3).  Outputs: du (nsys, n, d) and parameter gradients (nset, n, slots)
 * summed over the systems of each set (written, or added when accumulate = 1).  scratch: lpm_grad_scratch_bytes. */
int lpm_energy_vjp_f64(const lpm_lattice* lat, const double* u, const double* G, const double* Kn, const double* Tv,
                       int32_t coef_layout, const lpm_batch* batch, double* du, double* gKn, double* gTv,
                       int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream);
int lpm_stress_vjp_f64(const lpm_lattice* lat, const double* u, const double* Gsig, const double* Kn,
                       const double* Tv, int32_t coef_layout, const lpm_batch* batch, const double* l0, double V,
                       double* du, double* gKn, double* gTv, int32_t accumulate, void* scratch, size_t scratch_bytes,
                       void* stream);
/* VJP of f = K u on the SC lattice (the autograd pass of coarse3d/torch_lpm3d.py:81-83): du = K^T G for upstream G
 * (nsys, n, 3), exact also for bond parameters that are not symmetric, and the parameter gradients of sum G . K u.
 * The square lattice's exact Hessian is symmetric (use lpm_kmv_sq_* and lpm_bond_grad_sq): LPM_ERR_UNSUPPORTED. */
int lpm_kmv_vjp_f64(const lpm_lattice* lat, const double* u, const double* G, const double* Kn, const double* Tv,
                    int32_t coef_layout, const lpm_batch* batch, double* du, double* gKn, double* gTv,
                    int32_t accumulate, void* scratch, size_t scratch_bytes, void* stream);

/* ---------------------------------------------------------------------------------- AMG preconditioner */
/* Aggregation AMG of timing/t3d/amg3d.py (AMGGeom, AMG3D) for the SC operator on full boxes (FP32 coefficients,
 * packed LPM_LAYOUT_SOA; nx a multiple of 4), used as the preconditioner of an FP32 PCG and, through lpm_ir_amg, of
 * the mixed-precision solve.  Defaults (lpm_amg_default_opts) are the settings of timing/t3d/problems.py:19
 * (AMG_CFG): agg 3, coarse_max 1000, nu 1, W-cycles (gamma 2) below the finest level, 5 power iterations. */
typedef struct lpm_amg_opts {
    int32_t agg;          /* aggregate edge in sites (>= 3); the remainder joins the last chunk (rule "merge") */
    int32_t coarse_max;   /* the coarsest level is solved densely once 6 * nodes <= coarse_max */
    int32_t max_levels;   /* limit on coarse levels below level 1 (<= 8) */
    int32_t nu;           /* smoothing sweeps on the finest level before and after the coarse correction (1) */
    int32_t nu_c;         /* sweeps on the coarse levels (>= 1) */
    int32_t gamma;        /* cycle index on levels >= w_from (1 = V, 2 = W) */
    int32_t w_from;       /* first level with gamma cycles (levels counted from 1 below the finest) */
    int32_t power_its;    /* power iterations for rho(D^-1 A) of every smoothed level */
    double omega;         /* smoother weight omega / rho */
    int32_t rho0_per_box; /* 0: rho of the finest level from the first box of a set, reused for its other boxes
                             (timing/t3d/problems.py:126-128); 1: one estimate per box */
    int32_t reserved;
} lpm_amg_opts;

typedef struct lpm_amg lpm_amg; /* opaque: geometry, per-set hierarchies and solver state of one batch shape */

void lpm_amg_default_opts(lpm_amg_opts* opts);
/* Geometry of the hierarchy for a batch (host work and one device allocation, freed by lpm_amg_destroy).  boxes:
 * (nbox, 6) int32 free boxes lo x, y, z, hi x, y, z (inclusive site indices); box_of_mask (batch->nmask): the box of
 * DOF mask m -- system s is free exactly on the particles of box box_of_mask[s % nmask] (all three DOFs), as for
 * every load case of geom3d.prescribed.  One hierarchy per (coefficient set, box), as timing/t3d/problems.py:112-132
 * builds one per BC set.  Replaces amg3d.AMGGeom (timing/t3d/amg3d.py:440-497). */
int lpm_amg_create(const lpm_lattice* lat, const lpm_batch* batch, const int32_t* boxes, int32_t nbox,
                   const int32_t* box_of_mask, const lpm_amg_opts* opts, lpm_amg** out);
void lpm_amg_destroy(lpm_amg* amg);
/* Numeric setup for the batch's coefficient sets (replaces amg3d.AMG3D.__init__, timing/t3d/amg3d.py:522-570):
 * Kn32/Tv32 packed FP32 (nset, 18, n), copied into the handle (so the caller's arrays are free after the call, and
 * graphs of the handle's solves stay valid across setups); Minv32 the FP32 block-Jacobi inverse
 * (nset, n, 3, 3) of lpm_block_jacobi_f32.  Synchronises the stream. */
int lpm_amg_setup(lpm_amg* amg, const float* Kn32, const float* Tv32, const float* Minv32, void* stream);
/* rho of the finest level per (set, box estimate): (nset * nb) values, nb = nbox with rho0_per_box else 1.  set_rho0
 * replaces the estimates (amg3d.AMG3D's rho0 argument: a value shared by the BC sets of one specimen). */
int lpm_amg_get_rho0(const lpm_amg* amg, double* rho0_host);
int lpm_amg_set_rho0(lpm_amg* amg, const double* rho0_host, void* stream);
/* One preconditioner application z = B r for every system (amg3d.AMG3D.vcycle, timing/t3d/amg3d.py:609-637);
 * r, z: (nsys, n, 3) FP32, r is masked to the free box first. */
int lpm_amg_apply(lpm_amg* amg, const float* r, float* z, void* stream);
/* FP32 AMG-preconditioned CG from x = 0 (amg3d.AMG3D.pcg, timing/t3d/amg3d.py:639-668, batched with freezing):
 * b, x (nsys, n, 3) FP32; opts, outputs and stop rule as lpm_cg_batched_*. */
int lpm_amg_pcg_f32(lpm_amg* amg, const float* b, float* x, const lpm_cg_opts* opts, int32_t* iters, double* relres,
                    int32_t* status, void* stream);
/* Mixed-precision solve as lpm_ir_batched with the FP32 AMG-PCG as the inner solver (the handle's coefficients and
 * batch); workspace: lpm_ir_workspace_bytes(lat, batch, 0). */
int lpm_ir_amg(const lpm_lattice* lat, const double* Kn64, const double* Tv64, int32_t coef_layout64, lpm_amg* amg,
               const lpm_batch* batch, const uint8_t* mask, const double* b, double* x, const lpm_ir_opts* opts,
               void* workspace, size_t workspace_bytes, int32_t* iters, double* relres, int32_t* status,
               int32_t* outer_steps, void* stream);
/* Levels of a box (nlev: stencil levels below the finest, the last one dense), their grids (nlev, 3) and the
 * handle's device bytes. */
int lpm_amg_info(const lpm_amg* amg, int32_t box, int32_t* nlev, int32_t* grids, int64_t* device_bytes);
/* Level `level` (1..nlev) of the hierarchy (set, box) after setup, to host memory: A_host (nodes, 27, 6, 6) FP32
 * stencil rows as amg3d.AMG3D.A, rho_host its rho (0 for the dense level), fw_host (nsys) the finest-level smoother
 * weights omega / rho0; any output may be NULL.  Synchronises the device. */
int lpm_amg_get_level(const lpm_amg* amg, int32_t box, int32_t set, int32_t level, float* A_host, double* rho_host,
                      float* fw_host);

/* ------------------------------------------------------------------------------------------------- tuning */
/* Autotuner of the FP32 packed-coefficient SC operator used by the CG engines on full boxes: times its two variants
 * (0: Tv and Kn staged in shared memory, one CTA per SM; 1: lean, two CTAs per SM) with each z-chunk candidate (whole
 * box, 1/2, 1/3, ... of the planes, at least 8 planes per chunk) on zero vectors of the batch's shape, records the
 * fastest for (nx, ny, nz, pairs) in a process-wide table that later launches of that shape use, and returns it
 * (variant_out may be NULL).  Kn/Tv: packed FP32 coefficients (LPM_LAYOUT_SOA) of the batch's sets.  scratch:
 * lpm_kmv_scratch_bytes(lat, LPM_F32, nsys).  No reference counterpart (tuning of this library's tiles). */
int lpm_autotune_kmv(const lpm_lattice* lat, const lpm_batch* batch, const float* Kn, const float* Tv, void* scratch,
                     size_t scratch_bytes, int32_t* zchunk_out, int32_t* variant_out, void* stream);
/* Pins the operator's tiles for a batch shape instead of timing them (reproducible runs, tests): z planes per CTA
 * (1..nz, at most nz/8 chunks) and variant (0 or 1, as above).  No reference counterpart. */
int lpm_tune_kmv_set(const lpm_lattice* lat, const lpm_batch* batch, int32_t zchunk, int32_t variant);

/* --------------------------------------------------------------------------------------- parameter assembly */
/* Symmetric scatter of per-bond values to a (nspec, n, 18) parameter array (coarse3d/train3d.py:77-97, Scatter):
 * out[b, p_j, k_j] = out[b, q_j, k_j ^ 1] = vals[b, j] for the nb bonds of one group (q_j = -1: no second end).
 * out must hold the values of earlier groups (or zeros); later writes win, as index_put does. */
int lpm_bond_scatter_f64(int32_t nspec, int64_t n, int64_t nb, const int32_t* p, const int32_t* k, const int32_t* q,
                         const double* vals, double* out, void* stream);
/* Its adjoint: g[b, j] = G[b, p_j, k_j] + G[b, q_j, k_j ^ 1] (the autograd pass of Scatter for bonds written once). */
int lpm_bond_gather_sym_f64(int32_t nspec, int64_t n, int64_t nb, const int32_t* p, const int32_t* k,
                            const int32_t* q, const double* G, double* g, void* stream);
/* Smallest eigenvalue lam (nspec, n) and its unit eigenvector vec (nspec, n, 6 or 12) of every (particle, shell) group
 * bond Hessian of the stability penalty (coarse3d/train3d.py:119-137, group_penalty): H = diag(kn) + (tv 1^T +
 * 1 tv^T)/2 on the shell's in-box slots and 1e3 sc[b] on the diagonal of the others; Kn, Tv (nspec, n, 18) FP64 in the
 * reference layout, full SC boxes only. */
int lpm_group_eigmin_sc(const lpm_lattice* lat, int32_t nspec, const double* Kn, const double* Tv, const double* sc,
                        int32_t shell, double* lam, double* vec, void* stream);

/* ------------------------------------------------------------------------------------------------ geometry */
/* Neighbour table of a (possibly masked) box, identical to LatticeGeom.nbr / Lattice2D.nbr
 * (coarse3d/geom3d.py:38-65, coarse2d/lin2d.py:32-74): site_of (nx*ny*nz) int64 = particle id or -1,
 * sites (n) int64 = site of each particle; nbr (n, slots) int64 out. */
int lpm_build_nbr(int32_t dim, int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t* site_of,
                  const int64_t* sites, int64_t* nbr, void* stream);

/* Bond tables of specimens with voids on the full box (nx*ny*nz sites, all kept in the numbering): solid (nspec, n)
 * uint8 (1 = solid); nbr (nspec, n, slots) int32 out, slot k of site i = its grid neighbour q if both i and q are
 * solid, else -1.  This is the per-specimen bond validity gvalid & solid_i & solid_q of cement3d/torch_v1.py:37-45
 * (SCTV.set_mask); each table is the nbr of an lpm_lattice for that specimen's operator calls. */
int lpm_solid_nbr(int32_t dim, int32_t nx, int32_t ny, int32_t nz, int32_t nspec, const uint8_t* solid, int32_t* nbr,
                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LPM_B200_H */
