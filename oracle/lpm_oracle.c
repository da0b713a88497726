/*
 * lpm_oracle.c -- CPU oracle for the LPM linear solve.  TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C with OpenMP, the reference's FP64 CPU algorithms for the hot path, so that the GPU
 * library can be checked against them and timed beside them.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may call it; the product path (the CUDA library) never does.
 *
 * Parity pins: tests/test_oracle.py checks every function here against golden vectors produced by running the
 * reference itself (tests/golden/make_golden.py).
 *
 * Conventions (same as the reference): neighbour table nbr (N, NN) int64 with -1 for a missing bond; ndir (NN, d)
 * unit bond directions n_k = (x_i - x_q)/|x_i - x_q|; slots in reverse pairs (k, k^1); shell 0 = axial slots
 * (k < 6 in 3D, k < 4 in 2D), shell 1 = diagonal slots.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ============================================================================================================
 * 3D simple-cubic lattice, "code force" form
 * ============================================================================================================ */

/* dL_ik = n_k . (u_i - u_q)  */
static inline double sc_dl(const double *ndir, const double *u, i64 i, i64 q, int k)
{
    return ndir[3 * k] * (u[3 * i] - u[3 * q]) + ndir[3 * k + 1] * (u[3 * i + 1] - u[3 * q + 1]) +
           ndir[3 * k + 2] * (u[3 * i + 2] - u[3 * q + 2]);
}

/* Per-particle shell sums S_c = sum_{k in c} dL_ik and TS_c = sum_{k in c} Tv_ik dL_ik.
 * Follows coarse3d/lin3d.py:98-123 (k_shell_sums).  S, TS: (N, 2). */
void orc_sc_shell_sums(i64 N, const i64 *nbr, const double *ndir, const double *Tv, const double *u, double *S,
                       double *TS)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double s[2] = {0.0, 0.0}, t[2] = {0.0, 0.0};
        for (int k = 0; k < 18; ++k) {
            i64 q = nbr[18 * i + k];
            if (q < 0) continue;
            double d = sc_dl(ndir, u, i, q, k);
            int c = k < 6 ? 0 : 1;
            s[c] += d;
            t[c] += Tv[18 * i + k] * d;
        }
        S[2 * i] = s[0];
        S[2 * i + 1] = s[1];
        TS[2 * i] = t[0];
        TS[2 * i + 1] = t[1];
    }
}

/* Bond force F_ik = 2 Kn dL + (TS_i^c + TS_q^c)/2 + Tv (S_i^c + S_q^c)/2 (coarse3d/lin3d.py:152-167). */
void orc_sc_bond_forces(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv,
                        const double *u, double *dL, double *F)
{
    double *S = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    double *TS = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    orc_sc_shell_sums(N, nbr, ndir, Tv, u, S, TS);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        for (int k = 0; k < 18; ++k) {
            i64 q = nbr[18 * i + k];
            double d = 0.0, f = 0.0;
            if (q >= 0) {
                int c = k < 6 ? 0 : 1;
                d = sc_dl(ndir, u, i, q, k);
                f = 2.0 * Kn[18 * i + k] * d + 0.5 * (TS[2 * i + c] + TS[2 * q + c]) +
                    0.5 * Tv[18 * i + k] * (S[2 * i + c] + S[2 * q + c]);
            }
            if (dL) dL[18 * i + k] = d;
            F[18 * i + k] = f;
        }
    }
    free(S);
    free(TS);
}

/* out = K u, out_i = sum_k F_ik n_k (coarse3d/lin3d.py:126-149, k_apply). */
void orc_sc_apply(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *u,
                  double *out)
{
    double *S = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    double *TS = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    orc_sc_shell_sums(N, nbr, ndir, Tv, u, S, TS);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double o0 = 0.0, o1 = 0.0, o2 = 0.0;
        for (int k = 0; k < 18; ++k) {
            i64 q = nbr[18 * i + k];
            if (q < 0) continue;
            int c = k < 6 ? 0 : 1;
            double d = sc_dl(ndir, u, i, q, k);
            double f = 2.0 * Kn[18 * i + k] * d + 0.5 * (TS[2 * i + c] + TS[2 * q + c]) +
                       0.5 * Tv[18 * i + k] * (S[2 * i + c] + S[2 * q + c]);
            o0 += f * ndir[3 * k];
            o1 += f * ndir[3 * k + 1];
            o2 += f * ndir[3 * k + 2];
        }
        out[3 * i] = o0;
        out[3 * i + 1] = o1;
        out[3 * i + 2] = o2;
    }
    free(S);
    free(TS);
}

/* computeStress with the opp-flag surface rule (coarse3d/lin3d.py:170-210).  out (N, 6): xx yy zz yz xz xy. */
void orc_sc_stress(i64 N, const i64 *nbr, const double *ndir, const double *l0, const double *Kn, const double *Tv,
                   double V, const double *u, double *out)
{
    double *F = (double *)malloc(sizeof(double) * 18 * (size_t)N);
    orc_sc_bond_forces(N, nbr, ndir, Kn, Tv, u, NULL, F);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        int nb = 0;
        for (int k = 0; k < 18; ++k) nb += nbr[18 * i + k] >= 0;
        double s[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 18; ++k) {
            if (nbr[18 * i + k] < 0) continue;
            double of = (nb != 18 && nbr[18 * i + (k ^ 1)] < 0) ? 1.0 : 0.5;
            double a = of / V * l0[k] * F[18 * i + k];
            double n0 = ndir[3 * k], n1 = ndir[3 * k + 1], n2 = ndir[3 * k + 2];
            s[0] += a * n0 * n0;
            s[1] += a * n1 * n1;
            s[2] += a * n2 * n2;
            s[3] += a * n1 * n2;
            s[4] += a * n0 * n2;
            s[5] += a * n0 * n1;
        }
        for (int c = 0; c < 6; ++c) out[6 * i + c] = s[c];
    }
    free(F);
}

/* Particle energy U_i = 1/2 sum Kn dL^2 + 1/2 sum_c S_c TS_c (coarse3d/lin3d.py:213-236). */
void orc_sc_energy(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *u,
                   double *out)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double e = 0.0, s[2] = {0, 0}, t[2] = {0, 0};
        for (int k = 0; k < 18; ++k) {
            i64 q = nbr[18 * i + k];
            if (q < 0) continue;
            double d = sc_dl(ndir, u, i, q, k);
            int c = k < 6 ? 0 : 1;
            e += 0.5 * Kn[18 * i + k] * d * d;
            s[c] += d;
            t[c] += Tv[18 * i + k] * d;
        }
        out[i] = e + 0.5 * (s[0] * t[0] + s[1] * t[1]);
    }
}

/* 3x3 diagonal blocks of K (coarse3d/lin3d.py:239-269).  D: (N, 3, 3). */
void orc_sc_block_diag(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, double *D)
{
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < N; ++p) {
        double Dp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < 2; ++c) {
            int k0 = c == 0 ? 0 : 6, k1 = c == 0 ? 6 : 18;
            double T[3] = {0, 0, 0}, s[3] = {0, 0, 0};
            for (int a = k0; a < k1; ++a) {
                if (nbr[18 * p + a] < 0) continue;
                for (int d = 0; d < 3; ++d) {
                    T[d] += Tv[18 * p + a] * ndir[3 * a + d];
                    s[d] += ndir[3 * a + d];
                }
            }
            for (int d = 0; d < 3; ++d)
                for (int e = 0; e < 3; ++e) Dp[3 * d + e] += 0.5 * (T[d] * s[e] + s[d] * T[e]);
            for (int a = k0; a < k1; ++a) {
                i64 q = nbr[18 * p + a];
                if (q < 0) continue;
                int a2 = a ^ 1;
                double coef = Kn[18 * p + a] + Kn[18 * q + a2] + Tv[18 * q + a2];
                for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) Dp[3 * d + e] += coef * ndir[3 * a + d] * ndir[3 * a + e];
            }
        }
        memcpy(D + 9 * p, Dp, sizeof(Dp));
    }
}

/* Inverse by cofactors (coarse3d/lin3d.py:272-291). */
static void inv3(const double *A, double *out)
{
    double a = A[0], b = A[1], c = A[2], d = A[3], e = A[4], f = A[5], g = A[6], h = A[7], i = A[8];
    double co00 = e * i - f * h, co01 = -(d * i - f * g), co02 = d * h - e * g;
    double det = a * co00 + b * co01 + c * co02;
    out[0] = co00 / det;
    out[3] = co01 / det;
    out[6] = co02 / det;
    out[1] = -(b * i - c * h) / det;
    out[4] = (a * i - c * g) / det;
    out[7] = -(a * h - b * g) / det;
    out[2] = (b * f - c * e) / det;
    out[5] = -(a * f - c * d) / det;
    out[8] = (a * e - b * d) / det;
}

/* Block-Jacobi preconditioner M = D^-1 on free particles, 0 on fixed (coarse3d/lin3d.py:294-301). */
void orc_block_jacobi3(i64 N, const double *D, const uint8_t *free_, double *M)
{
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < N; ++p) {
        if (free_[p])
            inv3(D + 9 * p, M + 9 * p);
        else
            memset(M + 9 * p, 0, 9 * sizeof(double));
    }
}

/* Block-Jacobi PCG on the free particles (coarse3d/lin3d.py:464-518, _pcg).  b, x: (N,3), zero on fixed particles;
 * x is updated in place.  Stops when ||r|| <= tol ||b||, tested every iteration.  Returns the iteration count and
 * writes the relative residual. */
int orc_sc_pcg(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *M,
               const uint8_t *free_, const double *b, double *x, double tol, int maxit, double *relres)
{
    size_t n3 = 3 * (size_t)N;
    double *r = (double *)malloc(sizeof(double) * n3), *z = (double *)malloc(sizeof(double) * n3);
    double *p = (double *)malloc(sizeof(double) * n3), *Ap = (double *)malloc(sizeof(double) * n3);
    orc_sc_apply(N, nbr, ndir, Kn, Tv, x, Ap);
    double bn = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bn)
    for (i64 i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            r[3 * i + d] = free_[i] ? b[3 * i + d] - Ap[3 * i + d] : 0.0;
            bn += b[3 * i + d] * b[3 * i + d];
        }
    }
    bn = sqrt(bn);
    int it = 0;
    double rn = 0.0;
    if (bn == 0.0) {
        *relres = 0.0;
        free(r); free(z); free(p); free(Ap);
        return 0;
    }
    double rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz)
    for (i64 i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            const double *m = M + 9 * i + 3 * d;
            z[3 * i + d] = m[0] * r[3 * i] + m[1] * r[3 * i + 1] + m[2] * r[3 * i + 2];
        }
        for (int d = 0; d < 3; ++d) {
            p[3 * i + d] = z[3 * i + d];
            rz += r[3 * i + d] * z[3 * i + d];
        }
    }
    for (it = 1; it <= maxit; ++it) {
        orc_sc_apply(N, nbr, ndir, Kn, Tv, p, Ap);
        double pAp = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
        for (i64 i = 0; i < N; ++i)
            if (free_[i]) pAp += p[3 * i] * Ap[3 * i] + p[3 * i + 1] * Ap[3 * i + 1] + p[3 * i + 2] * Ap[3 * i + 2];
        double alpha = rz / pAp;
        rn = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rn)
        for (i64 i = 0; i < N; ++i) {
            if (!free_[i]) continue;
            for (int d = 0; d < 3; ++d) {
                x[3 * i + d] += alpha * p[3 * i + d];
                r[3 * i + d] -= alpha * Ap[3 * i + d];
            }
            rn += r[3 * i] * r[3 * i] + r[3 * i + 1] * r[3 * i + 1] + r[3 * i + 2] * r[3 * i + 2];
        }
        rn = sqrt(rn);
        if (rn <= tol * bn) break;
        double rz2 = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz2)
        for (i64 i = 0; i < N; ++i) {
            for (int d = 0; d < 3; ++d) {
                const double *m = M + 9 * i + 3 * d;
                z[3 * i + d] = m[0] * r[3 * i] + m[1] * r[3 * i + 1] + m[2] * r[3 * i + 2];
            }
            rz2 += r[3 * i] * z[3 * i] + r[3 * i + 1] * z[3 * i + 1] + r[3 * i + 2] * z[3 * i + 2];
        }
        double beta = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule(static)
        for (i64 j = 0; j < (i64)n3; ++j) p[j] = z[j] + beta * p[j];
    }
    if (it > maxit) it = maxit;
    *relres = rn / bn;
    free(r); free(z); free(p); free(Ap);
    return it;
}

/* Plain (unpreconditioned) CG from x (timing/t3d/cgplain.py:11-55, cg3). */
int orc_sc_cg(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const uint8_t *free_,
              const double *b, double *x, double tol, int maxit, double *relres)
{
    size_t n3 = 3 * (size_t)N;
    double *r = (double *)malloc(sizeof(double) * n3), *p = (double *)malloc(sizeof(double) * n3);
    double *Ap = (double *)malloc(sizeof(double) * n3);
    orc_sc_apply(N, nbr, ndir, Kn, Tv, x, Ap);
    double bn = 0.0, rr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bn, rr)
    for (i64 i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            double v = free_[i] ? b[3 * i + d] - Ap[3 * i + d] : 0.0;
            r[3 * i + d] = v;
            p[3 * i + d] = v;
            bn += b[3 * i + d] * b[3 * i + d];
            rr += v * v;
        }
    }
    bn = sqrt(bn);
    if (bn == 0.0) {
        *relres = 0.0;
        free(r); free(p); free(Ap);
        return 0;
    }
    int it = 0;
    for (it = 1; it <= maxit; ++it) {
        orc_sc_apply(N, nbr, ndir, Kn, Tv, p, Ap);
        double pAp = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
        for (i64 i = 0; i < N; ++i)
            if (free_[i]) pAp += p[3 * i] * Ap[3 * i] + p[3 * i + 1] * Ap[3 * i + 1] + p[3 * i + 2] * Ap[3 * i + 2];
        double alpha = rr / pAp, rn = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rn)
        for (i64 i = 0; i < N; ++i) {
            if (!free_[i]) continue;
            for (int d = 0; d < 3; ++d) {
                x[3 * i + d] += alpha * p[3 * i + d];
                r[3 * i + d] -= alpha * Ap[3 * i + d];
            }
            rn += r[3 * i] * r[3 * i] + r[3 * i + 1] * r[3 * i + 1] + r[3 * i + 2] * r[3 * i + 2];
        }
        if (sqrt(rn) <= tol * bn) {
            rr = rn;
            break;
        }
        double beta = rn / rr;
        rr = rn;
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < N; ++i) {
            if (!free_[i]) continue;
            for (int d = 0; d < 3; ++d) p[3 * i + d] = r[3 * i + d] + beta * p[3 * i + d];
        }
    }
    if (it > maxit) it = maxit;
    *relres = sqrt(rr) / bn;
    free(r); free(p); free(Ap);
    return it;
}

/* Per-slot derivatives of lam . K(Kn, Tv) u for the code-force operator (closed form of the autograd pass in
 * coarse3d/torch_lpm3d.py:170-175):
 *   d/dKn_ik = 2 dL(u)_ik (n_k . lam_i)
 *   d/dTv_ik = 1/2 dL(u)_ik S_i^c(lam) + 1/2 (S_i^c(u) + S_q^c(u)) (n_k . lam_i)
 * Zero on missing bonds.  gKn, gTv: (N, 18), positive sign (LinSolve returns the negatives). */
void orc_sc_grad(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *u,
                 const double *lam, double *gKn, double *gTv)
{
    (void)Kn;
    double *Su = (double *)malloc(sizeof(double) * 2 * (size_t)N), *TSu = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    double *Sl = (double *)malloc(sizeof(double) * 2 * (size_t)N), *TSl = (double *)malloc(sizeof(double) * 2 * (size_t)N);
    orc_sc_shell_sums(N, nbr, ndir, Tv, u, Su, TSu);
    orc_sc_shell_sums(N, nbr, ndir, Tv, lam, Sl, TSl);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        for (int k = 0; k < 18; ++k) {
            i64 q = nbr[18 * i + k];
            double gk = 0.0, gt = 0.0;
            if (q >= 0) {
                int c = k < 6 ? 0 : 1;
                double d = sc_dl(ndir, u, i, q, k);
                double nl = ndir[3 * k] * lam[3 * i] + ndir[3 * k + 1] * lam[3 * i + 1] + ndir[3 * k + 2] * lam[3 * i + 2];
                gk = 2.0 * d * nl;
                gt = 0.5 * d * Sl[2 * i + c] + 0.5 * (Su[2 * i + c] + Su[2 * q + c]) * nl;
            }
            gKn[18 * i + k] = gk;
            gTv[18 * i + k] = gt;
        }
    }
    free(Su); free(TSu); free(Sl); free(TSl);
}

/* ============================================================================================================
 * 2D square lattice, exact-Hessian ("g-form") operator of timing/t2d/solver2d.py
 * ============================================================================================================ */

static inline double sq_dl(const double *ndir, const double *u, i64 i, i64 q, int k)
{
    return ndir[2 * k] * (u[2 * i] - u[2 * q]) + ndir[2 * k + 1] * (u[2 * i + 1] - u[2 * q + 1]);
}

/* f = K u with g_ik = Kn dL + (Tv S_i^c + TS_i^c)/2 and f_j = sum_k (g_jk + g_{q, k^1}) n_k
 * (timing/t2d/solver2d.py:269-305, _kmv).  g: scratch (N, 8). */
void orc_sq_kmv(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *u,
                double *g, double *f)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double s[2] = {0, 0}, t[2] = {0, 0};
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            if (q < 0) continue;
            double d = sq_dl(ndir, u, i, q, k);
            g[8 * i + k] = d;
            int c = k < 4 ? 0 : 1;
            s[c] += d;
            t[c] += Tv[8 * i + k] * d;
        }
        for (int k = 0; k < 8; ++k) {
            if (nbr[8 * i + k] < 0) continue;
            int c = k < 4 ? 0 : 1;
            g[8 * i + k] = Kn[8 * i + k] * g[8 * i + k] + 0.5 * (Tv[8 * i + k] * s[c] + t[c]);
        }
    }
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < N; ++j) {
        double fx = 0.0, fy = 0.0;
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * j + k];
            if (q < 0) continue;
            double t = g[8 * j + k] + g[8 * q + (k ^ 1)];
            fx += t * ndir[2 * k];
            fy += t * ndir[2 * k + 1];
        }
        f[2 * j] = fx;
        f[2 * j + 1] = fy;
    }
}

/* Inverse 2x2 diagonal blocks, zero for fixed particles (timing/t2d/solver2d.py:308-346).  Binv: (N, 2, 2). */
void orc_sq_diag_inv(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv,
                     const uint8_t *fixed, double *Binv)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double *B = Binv + 4 * i;
        if (fixed[i]) {
            B[0] = B[1] = B[2] = B[3] = 0.0;
            continue;
        }
        double a00 = 0, a01 = 0, a11 = 0, m[2][2] = {{0, 0}, {0, 0}}, t[2][2] = {{0, 0}, {0, 0}};
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            if (q < 0) continue;
            double nx = ndir[2 * k], ny = ndir[2 * k + 1];
            int c = k < 4 ? 0 : 1;
            double w = Kn[8 * i + k] + Kn[8 * q + (k ^ 1)] + Tv[8 * q + (k ^ 1)];
            a00 += w * nx * nx;
            a01 += w * nx * ny;
            a11 += w * ny * ny;
            m[c][0] += nx;
            m[c][1] += ny;
            t[c][0] += Tv[8 * i + k] * nx;
            t[c][1] += Tv[8 * i + k] * ny;
        }
        for (int c = 0; c < 2; ++c) {
            a00 += t[c][0] * m[c][0];
            a01 += 0.5 * (t[c][0] * m[c][1] + m[c][0] * t[c][1]);
            a11 += t[c][1] * m[c][1];
        }
        double det = a00 * a11 - a01 * a01;
        B[0] = a11 / det;
        B[1] = -a01 / det;
        B[2] = -a01 / det;
        B[3] = a00 / det;
    }
}

/* Matrix-free 2x2 block-Jacobi PCG on a per-DOF mask (timing/t2d/solver2d.py:349-421, pcg_mf, one tolerance).
 * Returns the iteration count, or -1 when maxit was reached (the reference's snapshot marker). */
int orc_sq_pcg_mf(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *Binv,
                  const double *mask, const double *b, double *x, double tol, int maxit, double *relres)
{
    size_t n = 2 * (size_t)N;
    double *r = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n);
    double *g = (double *)malloc(sizeof(double) * 8 * (size_t)N);
    orc_sq_kmv(N, nbr, ndir, Kn, Tv, x, g, Ap);
    double bb = 0, rr = 0;
#pragma omp parallel for schedule(static) reduction(+ : bb, rr)
    for (i64 i = 0; i < (i64)n; ++i) {
        r[i] = (b[i] - Ap[i]) * mask[i];
        bb += b[i] * b[i];
        rr += r[i] * r[i];
    }
    double bn = sqrt(bb);
    int it = 0, done = sqrt(rr) <= tol * bn;
    if (!done) {
        double rz = 0;
#pragma omp parallel for schedule(static) reduction(+ : rz)
        for (i64 c = 0; c < N; ++c) {
            double a0 = r[2 * c], a1 = r[2 * c + 1];
            double z0 = Binv[4 * c] * a0 + Binv[4 * c + 1] * a1, z1 = Binv[4 * c + 2] * a0 + Binv[4 * c + 3] * a1;
            p[2 * c] = z0;
            p[2 * c + 1] = z1;
            rz += a0 * z0 + a1 * z1;
        }
        while (it < maxit) {
            orc_sq_kmv(N, nbr, ndir, Kn, Tv, p, g, Ap);
            double pAp = 0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
            for (i64 i = 0; i < (i64)n; ++i) {
                Ap[i] *= mask[i];
                pAp += p[i] * Ap[i];
            }
            double alpha = rz / pAp;
            rr = 0;
#pragma omp parallel for schedule(static) reduction(+ : rr)
            for (i64 i = 0; i < (i64)n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * Ap[i];
                rr += r[i] * r[i];
            }
            ++it;
            if (sqrt(rr) <= tol * bn) {
                done = 1;
                break;
            }
            double rzn = 0;
#pragma omp parallel for schedule(static) reduction(+ : rzn)
            for (i64 c = 0; c < N; ++c) {
                double a0 = r[2 * c], a1 = r[2 * c + 1];
                double z0 = Binv[4 * c] * a0 + Binv[4 * c + 1] * a1, z1 = Binv[4 * c + 2] * a0 + Binv[4 * c + 3] * a1;
                z[2 * c] = z0;
                z[2 * c + 1] = z1;
                rzn += a0 * z0 + a1 * z1;
            }
            double beta = rzn / rz;
            rz = rzn;
#pragma omp parallel for schedule(static)
            for (i64 i = 0; i < (i64)n; ++i) p[i] = z[i] + beta * p[i];
        }
    }
    *relres = bn > 0 ? sqrt(rr) / bn : 0.0;
    free(r); free(z); free(p); free(Ap); free(g);
    return done ? it : -1;
}

/* Plain CG on a per-DOF mask (timing/t2d/cg2plain.py:11-49, cg_mf).  Returns the iteration count. */
int orc_sq_cg_mf(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *mask,
                 const double *b, double *x, double tol, int maxit, double *relres)
{
    size_t n = 2 * (size_t)N;
    double *r = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
    double *Ap = (double *)malloc(sizeof(double) * n), *g = (double *)malloc(sizeof(double) * 8 * (size_t)N);
    orc_sq_kmv(N, nbr, ndir, Kn, Tv, x, g, Ap);
    double bb = 0, rr = 0;
#pragma omp parallel for schedule(static) reduction(+ : bb, rr)
    for (i64 i = 0; i < (i64)n; ++i) {
        r[i] = (b[i] - Ap[i]) * mask[i];
        p[i] = r[i];
        bb += b[i] * b[i];
        rr += r[i] * r[i];
    }
    double bn = sqrt(bb);
    int it = 0;
    double rlast = rr;
    if (!(sqrt(rr) <= tol * bn)) {
        while (it < maxit) {
            orc_sq_kmv(N, nbr, ndir, Kn, Tv, p, g, Ap);
            double pAp = 0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
            for (i64 i = 0; i < (i64)n; ++i) {
                Ap[i] *= mask[i];
                pAp += p[i] * Ap[i];
            }
            double alpha = rr / pAp, rn = 0;
#pragma omp parallel for schedule(static) reduction(+ : rn)
            for (i64 i = 0; i < (i64)n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * Ap[i];
                rn += r[i] * r[i];
            }
            ++it;
            rlast = rn;
            if (sqrt(rn) <= tol * bn) break;
            double beta = rn / rr;
            rr = rn;
#pragma omp parallel for schedule(static)
            for (i64 i = 0; i < (i64)n; ++i) p[i] = r[i] + beta * p[i];
        }
    }
    *relres = bn > 0 ? sqrt(rlast) / bn : 0.0;
    free(r); free(p); free(Ap); free(g);
    return it;
}

/* Particle stress (xx, yy, xy) with the opp-flag rule (timing/t2d/solver2d.py:220-256 == lin2d.stress). */
void orc_sq_stress(i64 N, const i64 *nbr, const double *ndir, const double *l0, const double *Kn, const double *Tv,
                   double V, const double *u, double *sig)
{
    double *S = (double *)malloc(sizeof(double) * 2 * (size_t)N), *TS = (double *)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double s[2] = {0, 0}, t[2] = {0, 0};
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            if (q < 0) continue;
            double d = sq_dl(ndir, u, i, q, k);
            int c = k < 4 ? 0 : 1;
            s[c] += d;
            t[c] += Tv[8 * i + k] * d;
        }
        S[2 * i] = s[0]; S[2 * i + 1] = s[1];
        TS[2 * i] = t[0]; TS[2 * i + 1] = t[1];
    }
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        int full = 1;
        for (int k = 0; k < 8; ++k) full &= nbr[8 * i + k] >= 0;
        double sxx = 0, syy = 0, sxy = 0;
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            if (q < 0) continue;
            int c = k < 4 ? 0 : 1;
            double d = sq_dl(ndir, u, i, q, k);
            double F = 2.0 * Kn[8 * i + k] * d + 0.5 * (TS[2 * i + c] + TS[2 * q + c]) +
                       0.5 * Tv[8 * i + k] * (S[2 * i + c] + S[2 * q + c]);
            double of = (full || nbr[8 * i + (k ^ 1)] >= 0) ? 0.5 : 1.0;
            double a = of / V * l0[k] * F;
            sxx += a * ndir[2 * k] * ndir[2 * k];
            syy += a * ndir[2 * k + 1] * ndir[2 * k + 1];
            sxy += a * ndir[2 * k] * ndir[2 * k + 1];
        }
        sig[3 * i] = sxx;
        sig[3 * i + 1] = syy;
        sig[3 * i + 2] = sxy;
    }
    free(S); free(TS);
}

/* Particle energy (coarse2d/lin2d.py:156-163). */
void orc_sq_energy(i64 N, const i64 *nbr, const double *ndir, const double *Kn, const double *Tv, const double *u,
                   double *out)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double e = 0, s[2] = {0, 0}, t[2] = {0, 0};
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            if (q < 0) continue;
            double d = sq_dl(ndir, u, i, q, k);
            int c = k < 4 ? 0 : 1;
            e += 0.5 * Kn[8 * i + k] * d * d;
            s[c] += d;
            t[c] += Tv[8 * i + k] * d;
        }
        out[i] = e + 0.5 * (s[0] * t[0] + s[1] * t[1]);
    }
}

/* Per-slot derivatives of lam^T K u for the exact-Hessian operator (closed form of the autograd pass through
 * coarse2d/torch_lpm.py:173-191 assemble + 34-51 SPDSolve.backward):
 *   d/dKn_ik = dL(lam)_ik dL(u)_ik,   d/dTv_ik = 1/2 [dL(lam)_ik S_i^c(u) + dL(u)_ik S_i^c(lam)]. */
void orc_sq_grad(i64 N, const i64 *nbr, const double *ndir, const double *u, const double *lam, double *gKn,
                 double *gTv)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < N; ++i) {
        double dlu[8], dll[8], su[2] = {0, 0}, sl[2] = {0, 0};
        for (int k = 0; k < 8; ++k) {
            i64 q = nbr[8 * i + k];
            dlu[k] = dll[k] = 0.0;
            if (q < 0) continue;
            dlu[k] = sq_dl(ndir, u, i, q, k);
            dll[k] = sq_dl(ndir, lam, i, q, k);
            su[k < 4 ? 0 : 1] += dlu[k];
            sl[k < 4 ? 0 : 1] += dll[k];
        }
        for (int k = 0; k < 8; ++k) {
            int c = k < 4 ? 0 : 1;
            int ok = nbr[8 * i + k] >= 0;
            gKn[8 * i + k] = ok ? dll[k] * dlu[k] : 0.0;
            gTv[8 * i + k] = ok ? 0.5 * (dll[k] * su[c] + dlu[k] * sl[c]) : 0.0;
        }
    }
}
