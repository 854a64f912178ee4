/*
 * CPU oracle for the MaZe_Poisson per-step MD hot path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the contract.  Citations are to the reference project
 * (Crivella/MaZe_Poisson) by path within that project.
 *
 * Conventions kept from the reference so results match bit for bit:
 *  - grids are n^3, idx = (i*n + j)*n + k, periodic in all three axes (the reference's
 *    x-halo slabs filled by mpi_grid_exchange_bot_top, library/src/mpi_base.c:186-197,
 *    are the same as wrapping i);
 *  - every sum is accumulated in the reference's order, products are rounded before they
 *    are added (built with -ffp-contract=off, see Makefile);
 *  - reductions are serial, i.e. the reference run with OMP_NUM_THREADS=1.
 *
 * Pointwise passes (the stencils, BLAS-1 updates, one colour of a red-black sweep on an
 * even grid, the grid transfers, the pair forces of each ion) run on several host threads
 * (ORACLE_THREADS, default all cores).  Each output value is still computed by one thread
 * in the serial order, and every sum across points (dot products, the pair energy) stays
 * serial in index order, so the results do not depend on the thread count.
 */
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define PI_D 3.14159265358979323846
#define KB_HARTREE 3.1668e-6 /* library/include/constants.h:10 */

static inline long wrap(long a, long n) { a %= n; return a < 0 ? a + n : a; }

/* Host threads for the pointwise passes: ORACLE_THREADS, else every core. */
static int orc_threads(void) {
    static int nt = 0;
    if (nt == 0) {
        const char *e = getenv("ORACLE_THREADS");
        int v = e ? atoi(e) : 0;
        nt = v > 0 ? v : omp_get_num_procs();
        if (nt < 1) nt = 1;
    }
    return nt;
}
/* Parallel only where the pass is large enough to pay for the threads. */
#define PAR_MIN 32768L
static inline long gidx(long i, long j, long k, long n) {
    return (wrap(i, n) * n + wrap(j, n)) * n + wrap(k, n);
}

/* ------------------------------------------------------------------------------------
 * BLAS-1 helpers (library/src/linalg.c:105-212, serial no-BLAS build)
 * ---------------------------------------------------------------------------------- */
static double dot(const double *a, const double *b, long m) {
    double s = 0.0;
    for (long t = 0; t < m; t++) s += a[t] * b[t];
    return s;
}
/* max |a|: exact, so the order of the comparisons does not matter */
static double amax(const double *a, long m) {
    double s = 0.0;
#pragma omp parallel for reduction(max : s) num_threads(orc_threads()) if (m >= PAR_MIN)
    for (long t = 0; t < m; t++) { double v = fabs(a[t]); if (v > s) s = v; }
    return s;
}
/* u += alpha * v  (linalg.c:153-159) */
static void axpy(double *u, const double *v, double alpha, long m) {
#pragma omp parallel for num_threads(orc_threads()) if (m >= PAR_MIN)
    for (long t = 0; t < m; t++) u[t] += alpha * v[t];
}
static void scal(double *x, double alpha, long m) {
#pragma omp parallel for num_threads(orc_threads()) if (m >= PAR_MIN)
    for (long t = 0; t < m; t++) x[t] *= alpha;
}
/* out = in * a, pointwise */
static void scaled_copy(double *out, const double *in, double a, long m) {
#pragma omp parallel for num_threads(orc_threads()) if (m >= PAR_MIN)
    for (long t = 0; t < m; t++) out[t] = in[t] * a;
}

/* ------------------------------------------------------------------------------------
 * 7-point Laplacian, no 1/h^2 (library/src/laplace.c:24-75).
 * Sum order: x+1, x-1, y+1, y-1, z+1, z-1, then minus 6*centre.
 * ---------------------------------------------------------------------------------- */
void orc_laplace(const double *u, double *out, int n) {
    long nn = (long)n * n;
#pragma omp parallel for num_threads(orc_threads()) if (nn * n >= PAR_MIN)
    for (long i = 0; i < n; i++) {
        const double *up = u + wrap(i + 1, n) * nn, *um = u + wrap(i - 1, n) * nn;
        const double *uc = u + i * nn;
        for (long j = 0; j < n; j++) {
            const double *rp = uc + wrap(j + 1, n) * n, *rm = uc + wrap(j - 1, n) * n;
            const double *r0 = uc + j * n;
            for (long k = 0; k < n; k++) {
                long kp = k + 1 < n ? k + 1 : 0, km = k > 0 ? k - 1 : n - 1;
                double s = up[j * n + k] + um[j * n + k];
                s = s + rp[k];
                s = s + rm[k];
                s = s + r0[kp];
                s = s + r0[km];
                out[i * nn + j * n + k] = s - r0[k] * 6.0;
            }
        }
    }
}

/* ------------------------------------------------------------------------------------
 * CG with implicit Jacobi preconditioner (library/src/plcg.c:28-90).
 * Stops when ||r||_inf <= tol (absolute) after the x/r update; at most n^2 iterations;
 * returns the 0-based iteration index at convergence or -1.  x may alias b.
 * ---------------------------------------------------------------------------------- */
int orc_conj_grad(const double *b, const double *x0, double *x, double tol, int n) {
    long m = (long)n * n * n, limit = (long)n * n, iter = 0;
    int res = -1;
    double *r = malloc(m * sizeof(double)), *p = malloc(m * sizeof(double));
    double *Ap = malloc(m * sizeof(double));
    orc_laplace(x0, r, n);
    axpy(r, b, -1.0, m);                       /* r = A x0 - b */
    if (x != x0) memcpy(x, x0, m * sizeof(double));
    scaled_copy(p, r, 1.0 / 6.0, m);
    double rv = -dot(r, p, m);
    while (iter < limit) {
        orc_laplace(p, Ap, n);
        double alpha = rv / dot(p, Ap, m);
        axpy(x, p, alpha, m);
        axpy(r, Ap, alpha, m);
        double rr = dot(r, r, m);
        if (amax(r, m) <= tol) { res = (int)iter; break; }
        double rnv = -rr / 6.0, beta = rnv / rv;
        rv = rnv;
        scal(p, beta, m);
        axpy(p, r, 1.0 / 6.0, m);
        iter++;
    }
    free(r); free(p); free(Ap);
    return res;
}

/* ------------------------------------------------------------------------------------
 * Multigrid pieces (library/src/multigrid.c)
 * ---------------------------------------------------------------------------------- */

/* Red-black Gauss-Seidel, red = (i+j+k) even first (multigrid.c:636-729). */
void orc_smooth_rbgs(const double *rhs, double *x, int n, int iters) {
    const double inv_diag = -1.0 / 6.0;
    /* on an even grid a point's six neighbours all have the other colour, so the points
       of one colour are independent; on an odd grid the wrap joins equal colours and the
       sweep stays serial */
    int par = (n % 2 == 0) && (long)n * n * n >= PAR_MIN;
    for (int it = 0; it < iters; it++)
        for (int colour = 0; colour < 2; colour++)
#pragma omp parallel for num_threads(orc_threads()) if (par)
            for (long i = 0; i < n; i++)
                for (long j = 0; j < n; j++)
                    for (long k = (i + j + colour) & 1; k < n; k += 2) {
                        double s = x[gidx(i - 1, j, k, n)] + x[gidx(i + 1, j, k, n)];
                        s = s + x[gidx(i, j - 1, k, n)];
                        s = s + x[gidx(i, j + 1, k, n)];
                        s = s + x[gidx(i, j, k - 1, n)];
                        s = s + x[gidx(i, j, k + 1, n)];
                        long c = (i * n + j) * n + k;
                        x[c] = (rhs[c] - s) * inv_diag;
                    }
}

/* 27-point full weighting onto (n/2)^3, coarse (I,J,K) <- fine (2I,2J,2K)
   (multigrid.c:523-594); centre 8, faces 4, edges 2, corners 1, /64. */
void orc_restrict27(const double *in, double *out, int n) {
    int nc = n / 2;
#define F(a, b, c) in[gidx(i + (a), j + (b), k + (c), n)]
#pragma omp parallel for num_threads(orc_threads()) if ((long)nc * nc * nc >= PAR_MIN / 8)
    for (long I = 0; I < nc; I++)
        for (long J = 0; J < nc; J++)
            for (long K = 0; K < nc; K++) {
                long i = 2 * I, j = 2 * J, k = 2 * K;
                double f = F(-1, 0, 0) + F(1, 0, 0);
                f = f + F(0, -1, 0); f = f + F(0, 1, 0);
                f = f + F(0, 0, -1); f = f + F(0, 0, 1);
                double e = F(1, 0, -1) + F(1, 0, 1);
                e = e + F(-1, 0, -1); e = e + F(-1, 0, 1);
                e = e + F(1, -1, 0);  e = e + F(1, 1, 0);
                e = e + F(-1, -1, 0); e = e + F(-1, 1, 0);
                e = e + F(0, -1, -1); e = e + F(0, -1, 1);
                e = e + F(0, 1, -1);  e = e + F(0, 1, 1);
                double c = F(1, 1, -1) + F(1, 1, 1);
                c = c + F(1, -1, -1);  c = c + F(1, -1, 1);
                c = c + F(-1, 1, -1);  c = c + F(-1, 1, 1);
                c = c + F(-1, -1, -1); c = c + F(-1, -1, 1);
                double v = 8.0 * F(0, 0, 0) + 4.0 * f;
                v = v + 2.0 * e;
                v = v + c;
                out[(I * nc + J) * nc + K] = v * (1.0 / 64.0);
            }
#undef F
}

/* Trilinear prolongation from nc^3 onto (2nc)^3 (multigrid.c:393-463). Weights are
   (1,0) on even fine indices and (0.5,0.5) on odd ones; 8 terms summed in the
   reference's order. */
void orc_prolong_trilinear(const double *in, double *out, int nc) {
    long nf = 2L * nc;
#pragma omp parallel for num_threads(orc_threads()) if (nf * nf * nf >= PAR_MIN)
    for (long i = 0; i < nf; i++) {
        double wi0 = (i & 1) ? 0.5 : 1.0, wi1 = (i & 1) ? 0.5 : 0.0;
        long i0 = i / 2, i1 = i0 + 1;
        for (long j = 0; j < nf; j++) {
            double wj0 = (j & 1) ? 0.5 : 1.0, wj1 = (j & 1) ? 0.5 : 0.0;
            long j0 = (j / 2) % nc, j1 = j0 + 1;
            for (long k = 0; k < nf; k++) {
                double wk0 = (k & 1) ? 0.5 : 1.0, wk1 = (k & 1) ? 0.5 : 0.0;
                long k0 = (k / 2) % nc, k1 = k0 + 1;
#define C(a, b, c) in[gidx(a, b, c, nc)]
                double s = C(i0, j0, k0) * wi0 * wj0 * wk0 + C(i1, j0, k0) * wi1 * wj0 * wk0;
                s = s + C(i0, j1, k0) * wi0 * wj1 * wk0;
                s = s + C(i1, j1, k0) * wi1 * wj1 * wk0;
                s = s + C(i0, j0, k1) * wi0 * wj0 * wk1;
                s = s + C(i1, j0, k1) * wi1 * wj0 * wk1;
                s = s + C(i0, j1, k1) * wi0 * wj1 * wk1;
                s = s + C(i1, j1, k1) * wi1 * wj1 * wk1;
#undef C
                out[(i * nf + j) * nf + k] = s;
            }
        }
    }
}

/* Coarse-level CG with a relative inf-norm stop (multigrid.c:13-96). */
int orc_cg_coarse(const double *b, double *x, int n, int maxit, double rtol) {
    long m = (long)n * n * n;
    double *r = malloc(m * sizeof(double)), *p = malloc(m * sizeof(double));
    double *Ap = malloc(m * sizeof(double));
    int k;
    orc_laplace(x, r, n);
    axpy(r, b, -1.0, m);
    scaled_copy(p, r, 1.0 / 6.0, m);
    double r0 = amax(r, m);
    if (r0 == 0.0) { free(r); free(p); free(Ap); return 0; }
    double rv = -dot(r, p, m);
    for (k = 0; k < maxit; ++k) {
        orc_laplace(p, Ap, n);
        double den = dot(p, Ap, m);
        if (fabs(den) < 1e-300) break;
        double alpha = rv / den;
        axpy(x, p, alpha, m);
        axpy(r, Ap, alpha, m);
        if (amax(r, m) <= rtol * r0) { ++k; break; }
        double rr = dot(r, r, m);
        double rnv = -rr / 6.0, beta = rnv / rv;
        rv = rnv;
        scal(p, beta, m);
        axpy(p, r, 1.0 / 6.0, m);
    }
    free(r); free(p); free(Ap);
    return k;
}

/* One V-cycle as the reference runs it: the recursion bottoms out at depth 1, so this is
   a two-level cycle -- sm RBGS sweeps, residual, 27-pt restriction, coarse CG (50 it,
   rtol 1e-5) from zero, trilinear prolongation, correction, sm RBGS sweeps
   (multigrid.c:99-168, 743-765; multigrid.h:4-7). Requires n/2 >= 16. */
void orc_mg_apply(const double *rhs, double *x, int n, int sm) {
    long m = (long)n * n * n;
    int nc = n / 2;
    long mc = (long)nc * nc * nc;
    if (nc < 16) { fprintf(stderr, "oracle multigrid: requires n/2 >= 16\n"); exit(1); }
    double *r = malloc(m * sizeof(double));
    double *rc = malloc(mc * sizeof(double)), *ec = calloc(mc, sizeof(double));
    orc_smooth_rbgs(rhs, x, n, sm);
    orc_laplace(x, r, n);
    scal(r, -1.0, m);
    axpy(r, rhs, 1.0, m);
    orc_restrict27(r, rc, n);
    orc_cg_coarse(rc, ec, nc, 50, 1e-5);
    orc_prolong_trilinear(ec, r, nc);
    axpy(x, r, 1.0, m);
    orc_smooth_rbgs(rhs, x, n, sm);
    free(r); free(rc); free(ec);
}

/* ------------------------------------------------------------------------------------
 * Preconditioned CG (library/src/plcg.c:104-166) with the explicit preconditioners:
 * Jacobi, out = -in/6 (precond_jacobi.c:8-14), one V-cycle with 5 sweeps warm-started from
 * the previous output (precond_mg.c:3-5), SSOR (orc_ssor_apply) and block Jacobi
 * (orc_blockjacobi_apply).  The preconditioner output buffer starts at zero.
 * ---------------------------------------------------------------------------------- */
static void apply_precond(int kind, const double *in, double *out, int n) {
    long m = (long)n * n * n;
    if (kind == 1) {
#pragma omp parallel for num_threads(orc_threads()) if (m >= PAR_MIN)
        for (long t = 0; t < m; t++) out[t] = -in[t] / 6.0;
    }
    else if (kind == 3) orc_ssor_apply(in, out, n);
    else if (kind == 4) orc_blockjacobi_apply(in, out, n);
    else orc_mg_apply(in, out, n, 5);
}

static int conj_grad_precond(const double *b, const double *x0, double *x, double tol, int n,
                             int kind) {
    long m = (long)n * n * n, limit = (long)n * n, iter = 0;
    int res = -1;
    double *r = malloc(m * sizeof(double)), *Ap = malloc(m * sizeof(double));
    double *v = calloc(m, sizeof(double)), *p = malloc(m * sizeof(double));
    orc_laplace(x0, r, n);
    axpy(r, b, -1.0, m);
    if (x != x0) memcpy(x, x0, m * sizeof(double));
    apply_precond(kind, r, v, n);
    scaled_copy(p, v, -1.0, m);
    double rv = dot(r, v, m);
    while (iter < limit) {
        orc_laplace(p, Ap, n);
        double alpha = rv / dot(p, Ap, m);
        axpy(x, p, alpha, m);
        axpy(r, Ap, alpha, m);
        if (amax(r, m) <= tol) { res = (int)iter; break; }
        apply_precond(kind, r, v, n);
        double rnv = dot(r, v, m), beta = rnv / rv;
        rv = rnv;
        scal(p, beta, m);
        axpy(p, v, -1.0, m);
        iter++;
    }
    free(r); free(Ap); free(v); free(p);
    return res;
}

/* ------------------------------------------------------------------------------------
 * SSOR preconditioner (library/src/precond_ssor.c:1240-1252 with the edge solves of
 * precond_ssor.c:172-957, omega = 1.75): a forward sweep in index order, each point
 * b_c = (b_c + its neighbours of smaller flat index, taken in the order x+1, x-1, y+1,
 * y-1, z+1, z-1) / (6 / omega); b *= -6; a backward sweep in reverse index order over the
 * neighbours of larger index, same order and divisor; b *= (2 - omega) / omega. The
 * periodic wrap decides which neighbours count: at i = n-1 the x+1 neighbour (i = 0) has a
 * smaller index, at i = 0 the x-1 neighbour (i = n-1) a larger one.
 * ---------------------------------------------------------------------------------- */
static void ssor_sweep(double *b, int n, int forward, double dc) {
    long m = (long)n * n * n;
    for (long t = 0; t < m; t++) {
        long c = forward ? t : m - 1 - t;
        long i = c / ((long)n * n), j = (c / n) % n, k = c % n;
        long nb[6] = {gidx(i + 1, j, k, n), gidx(i - 1, j, k, n), gidx(i, j + 1, k, n),
                      gidx(i, j - 1, k, n), gidx(i, j, k + 1, n), gidx(i, j, k - 1, n)};
        double v = b[c];
        for (int q = 0; q < 6; q++)
            if (forward ? nb[q] < c : nb[q] > c) v = v + b[nb[q]];
        b[c] = v / dc;
    }
}

void orc_ssor_apply(const double *in, double *out, int n) {
    const double omega = 1.75, dc = 6.0 / omega;
    long m = (long)n * n * n;
    if (out != in) memcpy(out, in, m * sizeof(double));
    ssor_sweep(out, n, 1, dc);
    scal(out, -6.0, m);
    ssor_sweep(out, n, 0, dc);
    scal(out, (2 - omega) / omega, m);
}

/* ------------------------------------------------------------------------------------
 * Block-Jacobi preconditioner (library/src/precond_blockjacobi.c): the grid is cut into
 * 10^3 blocks; the preconditioner multiplies each block, as a row of 1000 values in
 * (i, j, k) order, by the inverse of the 7-point Laplacian of one block with Dirichlet
 * edges (diagonal -6, +1 to the in-block neighbours; precond_blockjacobi.c:14-69). The
 * reference inverts that matrix with LAPACK's dgetrf + dgetri (linalg.c:16-35), which
 * this image does not have: here it is Gauss-Jordan elimination with partial pivoting,
 * the same LU-based inverse up to rounding (parity unpinned). The product is the
 * reference's non-BLAS dgemm (linalg.c:170-181): every output summed serially over l.
 * ---------------------------------------------------------------------------------- */
#define BJ_B 10
#define BJ_B3 (BJ_B * BJ_B * BJ_B)
static double *bj_inv = NULL;

static void bj_build(void) {
    if (bj_inv) return;
    int n = BJ_B3;
    double *a = calloc((size_t)n * n, sizeof(double)), *inv = calloc((size_t)n * n, sizeof(double));
    for (int i = 0; i < BJ_B; i++)
        for (int j = 0; j < BJ_B; j++)
            for (int k = 0; k < BJ_B; k++) {
                long r = (i * BJ_B + j) * BJ_B + k;
                a[r * n + r] = -6.0;
                if (i > 0) a[r * n + r - BJ_B * BJ_B] = 1.0;
                if (i < BJ_B - 1) a[r * n + r + BJ_B * BJ_B] = 1.0;
                if (j > 0) a[r * n + r - BJ_B] = 1.0;
                if (j < BJ_B - 1) a[r * n + r + BJ_B] = 1.0;
                if (k > 0) a[r * n + r - 1] = 1.0;
                if (k < BJ_B - 1) a[r * n + r + 1] = 1.0;
            }
    for (long r = 0; r < n; r++) inv[r * n + r] = 1.0;
    for (long c = 0; c < n; c++) {
        long piv = c;
        for (long r = c + 1; r < n; r++)
            if (fabs(a[r * n + c]) > fabs(a[piv * n + c])) piv = r;
        if (piv != c)
            for (long q = 0; q < n; q++) {
                double t = a[c * n + q]; a[c * n + q] = a[piv * n + q]; a[piv * n + q] = t;
                t = inv[c * n + q]; inv[c * n + q] = inv[piv * n + q]; inv[piv * n + q] = t;
            }
        double d = a[c * n + c];
        for (long q = 0; q < n; q++) { a[c * n + q] /= d; inv[c * n + q] /= d; }
        for (long r = 0; r < n; r++) {
            double f = a[r * n + c];
            if (r == c || f == 0.0) continue;
            for (long q = 0; q < n; q++) {
                a[r * n + q] -= f * a[c * n + q];
                inv[r * n + q] -= f * inv[c * n + q];
            }
        }
    }
    free(a);
    bj_inv = inv;
}

/* precond_blockjacobi_apply (precond_blockjacobi.c:173-206): n a multiple of 10 */
void orc_blockjacobi_apply(const double *in, double *out, int n) {
    if (n % BJ_B) {
        fprintf(stderr, "Error: The size of the input vector is not a multiple of the block size (1000)\n");
        exit(1);
    }
    bj_build();
    int nb = n / BJ_B;
    double *row = malloc(BJ_B3 * sizeof(double));
    for (long bi = 0; bi < nb; bi++)
        for (long bj = 0; bj < nb; bj++)
            for (long bk = 0; bk < nb; bk++) {
                for (int l = 0; l < BJ_B3; l++)
                    row[l] = in[((bi * BJ_B + l / 100) * n + bj * BJ_B + (l / 10) % 10) * n + bk * BJ_B + l % 10];
                for (int p = 0; p < BJ_B3; p++) {
                    double c = 0.0;
                    for (int l = 0; l < BJ_B3; l++) c += row[l] * bj_inv[(long)l * BJ_B3 + p];
                    out[((bi * BJ_B + p / 100) * n + bj * BJ_B + (p / 10) % 10) * n + bk * BJ_B + p % 10] = c;
                }
            }
    free(row);
}

/* the block inverse itself (1000 x 1000, row-major), for the tests */
void orc_blockjacobi_inverse(double *out) {
    bj_build();
    memcpy(out, bj_inv, (size_t)BJ_B3 * BJ_B3 * sizeof(double));
}

/* ------------------------------------------------------------------------------------
 * Poisson-Boltzmann variant: face dielectric arrays eps_x/y/z (eps_x[c] sits on the
 * face between point c and its +x neighbour), cell screening k2, the variable-
 * coefficient operator and its solvers, and the boundary forces.
 * ---------------------------------------------------------------------------------- */

/* Smooth switch across the transition shell, a in [0, 2w] (grid_general.c:213-216). */
static double pb_switch(double a, double w2, double w3) {
    return -(1 / (4 * w3)) * pow(a, 3) + (3 / (4 * w2)) * pow(a, 2);
}
/* d(switch)/da / switch (particles.c:407-418). */
static double pb_h_ratio(double rad, double w2, double w3) {
    return (-(3 / (4 * w3)) * pow(rad, 2) + (3 / (2 * w2)) * rad) /
           (-(1 / (4 * w3)) * pow(rad, 3) + (3 / (4 * w2)) * pow(rad, 2));
}
/* One coefficient at squared distance r2 from an ion: untouched outside r_s + w, scaled
   by the switch inside the shell, zero inside r_s - w (grid_general.c:207-222). */
static void pb_scale(double *v, double r2, double rp2, double rm2, double rs, double w, double w2,
                     double w3) {
    if (r2 >= rp2) return;
    if (r2 > rm2) *v *= pb_switch(sqrt(r2) - rs + w, w2, w3);
    else *v = 0.0;
}

/* grid_update_eps_and_k2 (grid_general.c:138-301): eps = eps_s - eps_int and k2 = kbar2,
   scaled ion by ion (in ion order) over each ion's box of +-(floor((r_s+w)/h)+1) points,
   then eps += eps_int. */
void orc_update_eps_k2(const double *pos, const double *radii, int np, int n, double h, double w,
                       double eps_s, double eps_int, double kbar2, double *eps_x, double *eps_y,
                       double *eps_z, double *k2) {
    long m = (long)n * n * n, n2 = (long)n * n;
    double w2 = w * w, w3 = w2 * w, hd2 = h / 2.0;
    for (long t = 0; t < m; t++) {
        eps_x[t] = (eps_s - eps_int); eps_y[t] = (eps_s - eps_int); eps_z[t] = (eps_s - eps_int);
        k2[t] = kbar2;
    }
    for (int p = 0; p < np; p++) {
        double rs = radii[p], px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
        double rp2 = pow(rs + w, 2), rm2 = pow(rs - w, 2);
        int range = (int)floor((rs + w) / h) + 1;
        int ix = (int)floor(px / h), iy = (int)floor(py / h), iz = (int)floor(pz / h);
        if (range >= n) { fprintf(stderr, "oracle: PB ion box wider than the grid\n"); exit(1); }
        for (int di = -range; di <= range; di++) {
            int i0 = ix + di;
            double dx = px - i0 * h, dx2 = dx * dx;
            i0 = (i0 + n) % n;
            if (i0 < 0 || i0 >= n) continue;
            long ib = (long)i0 * n2;
            for (int dj = -range; dj <= range; dj++) {
                int j0 = iy + dj;
                double dy = py - j0 * h, dy2 = dy * dy;
                long jb = (long)((j0 + n) % n) * n;
                for (int dk = -range; dk <= range; dk++) {
                    int k0 = iz + dk;
                    double dz = pz - k0 * h, dz2 = dz * dz;
                    long c = ib + jb + (k0 + n) % n;
                    pb_scale(&k2[c], dx2 + dy2 + dz2, rp2, rm2, rs, w, w2, w3);
                    double a = dx - hd2;
                    pb_scale(&eps_x[c], a * a + dy2 + dz2, rp2, rm2, rs, w, w2, w3);
                    a = dy - hd2;
                    pb_scale(&eps_y[c], dx2 + a * a + dz2, rp2, rm2, rs, w, w2, w3);
                    a = dz - hd2;
                    pb_scale(&eps_z[c], dx2 + dy2 + a * a, rp2, rm2, rs, w, w2, w3);
                }
            }
        }
    }
    for (long t = 0; t < m; t++) { eps_x[t] += eps_int; eps_y[t] += eps_int; eps_z[t] += eps_int; }
}

/* Variable-coefficient operator (laplace.c:77-145): faces x+, x-, y+, y-, z+, z- times
   their neighbours, minus centre times (sum of the six faces + k2). */
void orc_laplace_pb(const double *u, double *out, const double *ex, const double *ey,
                    const double *ez, const double *k2, int n) {
    for (long i = 0; i < n; i++)
        for (long j = 0; j < n; j++)
            for (long k = 0; k < n; k++) {
                long c = (i * n + j) * n + k;
                long xm = gidx(i - 1, j, k, n), ym = gidx(i, j - 1, k, n), zm = gidx(i, j, k - 1, n);
                double s = u[gidx(i + 1, j, k, n)] * ex[c] + u[xm] * ex[xm];
                s = s + u[gidx(i, j + 1, k, n)] * ey[c];
                s = s + u[ym] * ey[ym];
                s = s + u[gidx(i, j, k + 1, n)] * ez[c];
                s = s + u[zm] * ez[zm];
                double d = ex[c] + ex[xm];
                d = d + ey[c]; d = d + ey[ym]; d = d + ez[c]; d = d + ez[zm]; d = d + k2[c];
                out[c] = s - u[c] * d;
            }
}

/* conj_grad_pb (plcg.c:169-238): conj_grad with the PB operator, still the implicit
   1/6 Jacobi scaling. */
int orc_conj_grad_pb(const double *b, const double *x0, double *x, double tol, int n,
                     const double *ex, const double *ey, const double *ez, const double *k2) {
    long m = (long)n * n * n, limit = (long)n * n, iter = 0;
    int res = -1;
    double *r = malloc(m * sizeof(double)), *p = malloc(m * sizeof(double));
    double *Ap = malloc(m * sizeof(double));
    orc_laplace_pb(x0, r, ex, ey, ez, k2, n);
    axpy(r, b, -1.0, m);
    if (x != x0) memcpy(x, x0, m * sizeof(double));
    scaled_copy(p, r, 1.0 / 6.0, m);
    double rv = -dot(r, p, m);
    while (iter < limit) {
        orc_laplace_pb(p, Ap, ex, ey, ez, k2, n);
        double alpha = rv / dot(p, Ap, m);
        axpy(x, p, alpha, m);
        axpy(r, Ap, alpha, m);
        double rr = dot(r, r, m);
        if (amax(r, m) <= tol) { res = (int)iter; break; }
        double rnv = -rr / 6.0, beta = rnv / rv;
        rv = rnv;
        scal(p, beta, m);
        axpy(p, r, 1.0 / 6.0, m);
        iter++;
    }
    free(r); free(p); free(Ap);
    return res;
}

/* smooth_pb_rbgs (multigrid_pb.c:544-640): red ((i+j+k) even) then black; x = (sum of
   face * neighbour - rhs) / max(diag, 1e-14). */
void orc_smooth_pb(const double *rhs, double *x, int n, int iters, const double *ex,
                   const double *ey, const double *ez, const double *k2) {
    for (int it = 0; it < iters; it++)
        for (int colour = 0; colour < 2; colour++)
            for (long i = 0; i < n; i++)
                for (long j = 0; j < n; j++)
                    for (long k = (i + j + colour) & 1; k < n; k += 2) {
                        long c = (i * n + j) * n + k;
                        long xm = gidx(i - 1, j, k, n), ym = gidx(i, j - 1, k, n), zm = gidx(i, j, k - 1, n);
                        double d = ex[c] + ex[xm];
                        d = d + ey[c]; d = d + ey[ym]; d = d + ez[c]; d = d + ez[zm]; d = d + k2[c];
                        if (d < 1e-14) d = 1e-14;
                        double s = ex[c] * x[gidx(i + 1, j, k, n)] + ex[xm] * x[xm];
                        s = s + ey[c] * x[gidx(i, j + 1, k, n)];
                        s = s + ey[ym] * x[ym];
                        s = s + ez[c] * x[gidx(i, j, k + 1, n)];
                        s = s + ez[zm] * x[zm];
                        s = s - rhs[c];
                        x[c] = s / d;
                    }
}

/* restriction_eps (multigrid_pb.c:330-447): the coarse +axis face is the mean of the 2x2
   fine faces of that axis around it; axis 0 = x, 1 = y, 2 = z. */
void orc_restrict_eps(const double *in, double *out, int n, int axis) {
    int nc = n / 2;
    for (long I = 0; I < nc; I++)
        for (long J = 0; J < nc; J++)
            for (long K = 0; K < nc; K++) {
                long i = 2 * I, j = 2 * J, k = 2 * K;
                double s;
                if (axis == 0)
                    s = in[gidx(i, j, k, n)] + in[gidx(i, j, k + 1, n)] + in[gidx(i, j + 1, k, n)] +
                        in[gidx(i, j + 1, k + 1, n)];
                else if (axis == 1)
                    s = in[gidx(i, j, k, n)] + in[gidx(i, j, k + 1, n)] + in[gidx(i + 1, j, k, n)] +
                        in[gidx(i + 1, j, k + 1, n)];
                else
                    s = in[gidx(i, j, k, n)] + in[gidx(i + 1, j, k, n)] + in[gidx(i, j + 1, k, n)] +
                        in[gidx(i + 1, j + 1, k, n)];
                out[(I * nc + J) * nc + K] = s * 0.25;
            }
}

/* restriction_k2screen (multigrid_pb.c:459-527) on one process (n_start = 0): coarse
   (I,J,K) is the mean of the fine cube at i in {2I+1, 2I+2}, j in {2J, 2J+1},
   k in {2K, 2K+1}. */
void orc_restrict_k2(const double *in, double *out, int n) {
    int nc = n / 2;
    for (long I = 0; I < nc; I++)
        for (long J = 0; J < nc; J++)
            for (long K = 0; K < nc; K++) {
                long i = 2 * I + 1, j = 2 * J, k = 2 * K;
                double s = in[gidx(i, j, k, n)] + in[gidx(i, j, k + 1, n)] + in[gidx(i, j + 1, k, n)] +
                           in[gidx(i, j + 1, k + 1, n)] + in[gidx(i + 1, j, k, n)] +
                           in[gidx(i + 1, j, k + 1, n)] + in[gidx(i + 1, j + 1, k, n)] +
                           in[gidx(i + 1, j + 1, k + 1, n)];
                out[(I * nc + J) * nc + K] = (1.0 / 8.0) * s;
            }
}

/* cg_coarse_pb (multigrid_pb.c:16-97): unpreconditioned CG, relative inf-norm stop. */
int orc_cg_coarse_pb(const double *b, double *x, int n, int maxit, double rtol, const double *ex,
                     const double *ey, const double *ez, const double *k2) {
    long m = (long)n * n * n;
    double *r = malloc(m * sizeof(double)), *p = malloc(m * sizeof(double));
    double *Ap = malloc(m * sizeof(double));
    int k;
    orc_laplace_pb(x, r, ex, ey, ez, k2, n);
    axpy(r, b, -1.0, m);
    for (long t = 0; t < m; t++) p[t] = r[t] * -1.0;
    double r0 = amax(r, m);
    if (r0 == 0.0) { free(r); free(p); free(Ap); return 0; }
    double rr = dot(r, r, m);
    for (k = 0; k < maxit; ++k) {
        orc_laplace_pb(p, Ap, ex, ey, ez, k2, n);
        double den = dot(p, Ap, m);
        if (fabs(den) < 1e-300) break;
        double alpha = rr / den;
        axpy(x, p, alpha, m);
        axpy(r, Ap, alpha, m);
        if (amax(r, m) <= rtol * r0) { ++k; break; }
        double rn = dot(r, r, m), beta = rn / rr;
        rr = rn;
        scal(p, beta, m);
        axpy(p, r, -1.0, m);
    }
    free(r); free(p); free(Ap);
    return k;
}

/* v_cycle_pb at depth 0 (multigrid_pb.c:270-328): sm PB-RBGS iterations, residual,
   27-pt restriction, face / cell restrictions of eps and k2, coarse PB CG (50 it, rtol
   1e-5) from zero, trilinear prolongation, correction, sm iterations. n/2 >= 16. */
void orc_mg_pb_apply(const double *rhs, double *x, int n, int sm, const double *ex,
                     const double *ey, const double *ez, const double *k2) {
    long m = (long)n * n * n;
    int nc = n / 2;
    long mc = (long)nc * nc * nc;
    if (nc < 16) { fprintf(stderr, "oracle multigrid: requires n/2 >= 16\n"); exit(1); }
    double *r = malloc(m * sizeof(double));
    double *rc = malloc(mc * sizeof(double)), *ec = calloc(mc, sizeof(double));
    double *cx = malloc(mc * sizeof(double)), *cy = malloc(mc * sizeof(double));
    double *cz = malloc(mc * sizeof(double)), *ck = malloc(mc * sizeof(double));
    orc_smooth_pb(rhs, x, n, sm, ex, ey, ez, k2);
    orc_laplace_pb(x, r, ex, ey, ez, k2, n);
    scal(r, -1.0, m);
    axpy(r, rhs, 1.0, m);
    orc_restrict27(r, rc, n);
    orc_restrict_eps(ex, cx, n, 0);
    orc_restrict_eps(ey, cy, n, 1);
    orc_restrict_eps(ez, cz, n, 2);
    orc_restrict_k2(k2, ck, n);
    orc_cg_coarse_pb(rc, ec, nc, 50, 1e-5, cx, cy, cz, ck);
    orc_prolong_trilinear(ec, r, nc);
    axpy(x, r, 1.0, m);
    orc_smooth_pb(rhs, x, n, sm, ex, ey, ez, k2);
    free(r); free(rc); free(ec); free(cx); free(cy); free(cz); free(ck);
}

/* particles_compute_forces_pb (particles.c:420-775): over each ion's box of
   +-(floor((r_s+w)/h)+2) points, in the shell r_s - w < r < r_s + w around the point
   (ionic boundary, k2 phi^2) and around each of its six faces (dielectric boundary,
   (eps_face - eps_int) * dphi * phi, and non-polar, eps gradient direction), summed
   ion by ion in loop order; then scaled by h/(8 pi), h/(8 pi) and
   -gamma_np h / (eps_s - eps_int). */
void orc_forces_pb(const double *pos, const double *radii, int np, int n, double h, double w,
                   double eps_s, double eps_int, double gamma_np, int nonpolar, const double *phi,
                   const double *ex, const double *ey, const double *ez, const double *k2,
                   double *fdb, double *fib, double *fnp) {
    double w2 = w * w, w3 = w2 * w, hd2 = h / 2.0;
    long v = 3L * np;
    memset(fdb, 0, v * sizeof(double)); memset(fib, 0, v * sizeof(double));
    memset(fnp, 0, v * sizeof(double));
    for (int p = 0; p < np; p++) {
        double *db = fdb + 3 * p, *ib = fib + 3 * p, *nq = fnp + 3 * p;
        double rs = radii[p], px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
        double rp2 = pow(rs + w, 2), rm2 = pow(rs - w, 2);
        int range = (int)floor((rs + w) / h) + 2;
        int ix = (int)floor(px / h), iy = (int)floor(py / h), iz = (int)floor(pz / h);
        if (range >= n) { fprintf(stderr, "oracle: PB ion box wider than the grid\n"); exit(1); }
        for (int di = -range; di <= range; di++) {
            int i = ix + di;
            double dx = px - i * h, dx2 = dx * dx;
            i = (i + n) % n;
            for (int dj = -range; dj <= range; dj++) {
                int j = iy + dj;
                double dy = py - j * h, dy2 = dy * dy;
                j = (j + n) % n;
                for (int dk = -range; dk <= range; dk++) {
                    int k = iz + dk;
                    double dz = pz - k * h, dz2 = dz * dz;
                    k = (k + n) % n;
                    long c = gidx(i, j, k, n);
                    long fx = gidx(i + 1, j, k, n), fy = gidx(i, j + 1, k, n), fz = gidx(i, j, k + 1, n);
                    long bx = gidx(i - 1, j, k, n), by = gidx(i, j - 1, k, n), bz = gidx(i, j, k - 1, n);
                    double exc = ex[c], eyc = ey[c], ezc = ez[c];
                    double exb = ex[bx], eyb = ey[by], ezb = ez[bz];
                    double ddx = exc - exb, ddy = eyc - eyb, ddz = ezc - ezb;
                    double dn = sqrt(ddx * ddx + ddy * ddy + ddz * ddz) / h;
                    double ig = (dn > 0.0) ? 1.0 / dn : 0.0;
                    double pc = phi[c];
                    double r2 = dx2 + dy2 + dz2, r1, rx, ry, rz, hr, a, g, dphi;
                    if (r2 < rp2 && r2 > rm2) {                      /* centre: ionic boundary */
                        r1 = sqrt(r2) + 1E-12;
                        rx = dx / r1; ry = dy / r1; rz = dz / r1;
                        hr = pb_h_ratio(r1 - rs + w, w2, w3);
                        a = k2[c] * pc * pc * hr;
                        ib[0] += a * rx; ib[1] += a * ry; ib[2] += a * rz;
                    }
                    /* six faces: (offset along the axis, sign of the non-polar term,
                       face coefficient, neighbour, gradient component) */
                    for (int f = 0; f < 6; f++) {
                        int axis = f / 2, fwd = f & 1;
                        double o = fwd ? -hd2 : hd2;
                        double ux = dx, uy = dy, uz = dz;
                        if (axis == 0) { ux = dx + o; r2 = ux * ux + dy2 + dz2; g = ig * ddx; }
                        else if (axis == 1) { uy = dy + o; r2 = dx2 + uy * uy + dz2; g = ig * ddy; }
                        else { uz = dz + o; r2 = dx2 + dy2 + uz * uz; g = ig * ddz; }
                        if (!(r2 < rp2 && r2 > rm2)) continue;
                        r1 = sqrt(r2) + 1E-12;
                        rx = ux / r1; ry = uy / r1; rz = uz / r1;
                        hr = pb_h_ratio(r1 - rs + w, w2, w3);
                        double ef = axis == 0 ? (fwd ? exc : exb) : axis == 1 ? (fwd ? eyc : eyb) : (fwd ? ezc : ezb);
                        long nb = axis == 0 ? (fwd ? fx : bx) : axis == 1 ? (fwd ? fy : by) : (fwd ? fz : bz);
                        a = (ef - eps_int) * hr;
                        dphi = phi[nb] - pc;
                        db[0] -= a * dphi * pc * rx; db[1] -= a * dphi * pc * ry; db[2] -= a * dphi * pc * rz;
                        if (nonpolar) {
                            if (fwd) { nq[0] += a * g * rx; nq[1] += a * g * ry; nq[2] += a * g * rz; }
                            else { nq[0] -= a * g * rx; nq[1] -= a * g * ry; nq[2] -= a * g * rz; }
                        }
                    }
                }
            }
        }
    }
    double cdb = h / (8.0 * PI_D), cnp = -gamma_np * h / (eps_s - eps_int);
    scal(fdb, cdb, v);
    scal(fib, cdb, v);
    scal(fnp, cnp, v);
}

/* ------------------------------------------------------------------------------------
 * Particle kernels
 * ---------------------------------------------------------------------------------- */

/* CIC weight (charges.c:8-14) with the minimum image over L = n*h. */
static inline double w_cic(double x, double L, double h) {
    x = fabs(x - round(x / L) * L);
    if (x >= h) return 0.0;
    return 1.0 - x / h;
}

void orc_cic_neighbors(const double *pos, int np, int n, double h, int64_t *nbr);

/* Quadratic and cubic B-spline weights (charges.c:16-38), with the reference's own pow()
   calls so that the oracle reproduces glibc's rounding. */
static double w_spl_quadr(double x, double L, double h) {
    x = fabs(x - round(x / L) * L) / h;
    if (x < 0.5) return 0.75 - x * x;
    if (x < 1.5) return 0.5 * pow((1.5 - x), 2);
    return 0.0;
}
static double w_spl_cubic(double x, double L, double h) {
    x = fabs(x - round(x / L) * L) / h;
    if (x < 1) return (4.0 - 6.0 * pow(x, 2) + 3.0 * pow(x, 3)) / 6.0;
    if (x < 2) return pow(2 - x, 3) / 6.0;
    return 0.0;
}
static double w_cic_fn(double x, double L, double h) { return w_cic(x, L, h); }

typedef double (*weight_fn)(double, double, double);
static weight_fn scheme_weight(int cas) {
    return cas == 1 ? w_spl_quadr : (cas == 2 ? w_spl_cubic : w_cic_fn);
}
static int scheme_points(int cas) { return cas == 0 ? 8 : 64; }

/* 4 x 4 x 4 points around floor(pos/h), offsets -1..2 nested a (x), b (y), c (z), each
   wrapped as (base + off + n) % n (particles.c:348-385). */
void orc_spline_neighbors(const double *pos, int np, int n, double h, int64_t *nbr) {
    for (long p = 0; p < np; p++) {
        long b[3];
        for (int d = 0; d < 3; d++) b[d] = (long)(int)floor(pos[3 * p + d] / h);
        long o = p * 64 * 3;
        for (int a = -1; a <= 2; a++)
            for (int bb = -1; bb <= 2; bb++)
                for (int cc = -1; cc <= 2; cc++) {
                    nbr[o++] = wrap(b[0] + a + n, n);
                    nbr[o++] = wrap(b[1] + bb + n, n);
                    nbr[o++] = wrap(b[2] + cc + n, n);
                }
    }
}

/* Zero q, then scatter chg*w over each ion's `nnb` stencil points in ion order
   (charges.c:100-144). Returns the total spread charge. */
static double spread_scheme(const double *pos, const double *chg, const int64_t *nbr, int nnb, int np,
                            int n, double h, double *q, weight_fn g) {
    double L = n * h, tot = 0.0;
    memset(q, 0, (size_t)n * n * n * sizeof(double));
    for (long p = 0; p < np; p++) {
        const int64_t *nb = nbr + p * nnb * 3;
        for (int c = 0; c < nnb; c++) {
            long a = nb[3 * c], b = nb[3 * c + 1], e = nb[3 * c + 2];
            double w = g(pos[3 * p] - a * h, L, h) * g(pos[3 * p + 1] - b * h, L, h);
            w = w * g(pos[3 * p + 2] - e * h, L, h);
            double u = chg[p] * w;
            tot += u;
            q[(a * n + b) * n + e] += u;
        }
    }
    return tot;
}

/* Field force by central differences of phi at each ion's stencil points
   (forces.c:26-100). Returns the sum of the stencil charges. */
static double force_scheme(const double *phi, const int64_t *nbr, int nnb, const double *chg,
                           const double *pos, int np, int n, double h, double *f, weight_fn g) {
    double L = n * h, h2 = 2.0 * h, sq = 0.0;
    for (long p = 0; p < np; p++) {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        const int64_t *nb = nbr + p * nnb * 3;
        for (int c = 0; c < nnb; c++) {
            long i = nb[3 * c], j = nb[3 * c + 1], k = nb[3 * c + 2];
            double qc = chg[p] * g(pos[3 * p] - i * h, L, h);
            qc = qc * g(pos[3 * p + 1] - j * h, L, h);
            qc = qc * g(pos[3 * p + 2] - k * h, L, h);
            sq += qc;
            fx += qc * ((phi[gidx(i - 1, j, k, n)] - phi[gidx(i + 1, j, k, n)]) / h2);
            fy += qc * ((phi[gidx(i, j - 1, k, n)] - phi[gidx(i, j + 1, k, n)]) / h2);
            fz += qc * ((phi[gidx(i, j, k - 1, n)] - phi[gidx(i, j, k + 1, n)]) / h2);
        }
        f[3 * p] = fx; f[3 * p + 1] = fy; f[3 * p + 2] = fz;
    }
    return sq;
}

/* Spreading / field force for scheme cas (0 CIC, 1 SPL_QUADR, 2 SPL_CUBIC) with the
   scheme's neighbour list built inside; nbr (np * points * 3) receives it if not null. */
double orc_spread_scheme(const double *pos, const double *chg, int np, int n, double h, int cas,
                         double *q, int64_t *nbr_out) {
    int nnb = scheme_points(cas);
    int64_t *nbr = nbr_out ? nbr_out : malloc((size_t)np * nnb * 3 * sizeof(int64_t));
    if (cas == 0) orc_cic_neighbors(pos, np, n, h, nbr);
    else orc_spline_neighbors(pos, np, n, h, nbr);
    double t = spread_scheme(pos, chg, nbr, nnb, np, n, h, q, scheme_weight(cas));
    if (!nbr_out) free(nbr);
    return t;
}
double orc_force_scheme(const double *phi, const double *chg, const double *pos, int np, int n, double h,
                        int cas, double *f) {
    int nnb = scheme_points(cas);
    int64_t *nbr = malloc((size_t)np * nnb * 3 * sizeof(int64_t));
    if (cas == 0) orc_cic_neighbors(pos, np, n, h, nbr);
    else orc_spline_neighbors(pos, np, n, h, nbr);
    double s = force_scheme(phi, nbr, nnb, chg, pos, np, n, h, f, scheme_weight(cas));
    free(nbr);
    return s;
}

/* Base cell floor(pos/h) and its 8 wrapped corners in the reference's order
   (particles.c:297-346). A base index outside [0,n) (a position at or beyond the box
   edge, where the reference indexes out of bounds) is wrapped. */
void orc_cic_neighbors(const double *pos, int np, int n, double h, int64_t *nbr) {
    static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                  {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
    for (long p = 0; p < np; p++) {
        long b[3];
        for (int d = 0; d < 3; d++) b[d] = wrap((long)(int)floor(pos[3 * p + d] / h), n);
        for (int c = 0; c < 8; c++)
            for (int d = 0; d < 3; d++)
                nbr[(p * 8 + c) * 3 + d] = off[c][d] ? (b[d] + 1) % n : b[d];
    }
}

/* Zero q, then scatter chg*w over the 8 corners in ion order (charges.c:100-144).
   Returns the total spread charge. */
double orc_spread_cic(const double *pos, const double *chg, const int64_t *nbr, int np, int n,
                      double h, double *q) {
    double L = n * h, tot = 0.0;
    memset(q, 0, (size_t)n * n * n * sizeof(double));
    for (long p = 0; p < np; p++) {
        const int64_t *nb = nbr + p * 24;
        for (int c = 0; c < 8; c++) {
            long a = nb[3 * c], b = nb[3 * c + 1], e = nb[3 * c + 2];
            double w = w_cic(pos[3 * p] - a * h, L, h) * w_cic(pos[3 * p + 1] - b * h, L, h);
            w = w * w_cic(pos[3 * p + 2] - e * h, L, h);
            double u = chg[p] * w;
            tot += u;
            q[(a * n + b) * n + e] += u;
        }
    }
    return tot;
}

/* Field force by central differences of phi at the 8 CIC corners (forces.c:26-100). */
double orc_force_fd(const double *phi, const int64_t *nbr, const double *chg, const double *pos,
                    int np, int n, double h, double *f) {
    double L = n * h, h2 = 2.0 * h, sq = 0.0;
    for (long p = 0; p < np; p++) {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        const int64_t *nb = nbr + p * 24;
        for (int c = 0; c < 8; c++) {
            long i = nb[3 * c], j = nb[3 * c + 1], k = nb[3 * c + 2];
            double qc = chg[p] * w_cic(pos[3 * p] - i * h, L, h);
            qc = qc * w_cic(pos[3 * p + 1] - j * h, L, h);
            qc = qc * w_cic(pos[3 * p + 2] - k * h, L, h);
            sq += qc;
            fx += qc * ((phi[gidx(i - 1, j, k, n)] - phi[gidx(i + 1, j, k, n)]) / h2);
            fy += qc * ((phi[gidx(i, j - 1, k, n)] - phi[gidx(i, j + 1, k, n)]) / h2);
            fz += qc * ((phi[gidx(i, j, k - 1, n)] - phi[gidx(i, j, k + 1, n)]) / h2);
        }
        f[3 * p] = fx; f[3 * p + 1] = fy; f[3 * p + 2] = fz;
    }
    return sq;
}

/* Per type-pair Tosi-Fumi table [A,B,C,D,sigma,alpha,beta] with the shifted-force
   constants at r_cut = L/2 (particles.c:181-228). The reference stores the same seven
   numbers per ion pair (7*N^2 doubles); they depend only on the two types. */
void orc_tf_table(const double *pp, int ntyp, double L, double *tab) {
    double rc = L / 2.0, rc6 = pow(rc, 6), rc7 = rc6 * rc, rc8 = rc7 * rc, rc9 = rc8 * rc;
    for (int t = 0; t < ntyp * ntyp; t++) {
        double A = pp[5 * t], B = pp[5 * t + 1], C = pp[5 * t + 2], D = pp[5 * t + 3],
               s = pp[5 * t + 4];
        double vs = A * exp(B * (s - rc)) - C / rc6 - D / rc8;
        double al = A * B * exp(B * (s - rc)) - 6 * C / rc7 - 8 * D / rc9;
        double be = -vs - al * rc;
        double *o = tab + 7 * t;
        o[0] = A; o[1] = B; o[2] = C; o[3] = D; o[4] = s; o[5] = al; o[6] = be;
    }
}

/* All-pairs shifted-force Tosi-Fumi, minimum image, skip r > r_cut, both orders summed
   over j ascending (forces.c:112-186). Returns half the summed pair energy.
   Each ion's force is its own serial sum over j, so ions run on several threads; the
   pair energies of a block of rows are kept in row order and added to the running total
   serially, ion by ion and j ascending, which is the reference's single-thread order. */
double orc_tf_forces(const double *pos, const int32_t *types, const double *tab, int ntyp, int np,
                     double L, double rcut, double *f) {
    const long rows = 64;
    double en = 0.0;
    double *ebuf = malloc((size_t)rows * (np > 0 ? np : 1) * sizeof(double));
    long *ecnt = malloc(rows * sizeof(long));
    for (long i0 = 0; i0 < np; i0 += rows) {
        long i1 = i0 + rows < np ? i0 + rows : np;
#pragma omp parallel for schedule(dynamic, 1) num_threads(orc_threads()) if ((long)np >= 512)
        for (long i = i0; i < i1; i++) {
            double fx = 0.0, fy = 0.0, fz = 0.0;
            double *erow = ebuf + (i - i0) * np;
            long ne = 0;
            for (long j = 0; j < np; j++) {
                if (i == j) continue;
                double d[3], r = 0.0;
                for (int a = 0; a < 3; a++) {
                    double x = pos[3 * i + a] - pos[3 * j + a];
                    x -= L * round(x / L);
                    d[a] = x;
                    r = (a == 0) ? x * x : r + x * x;
                }
                r = sqrt(r);
                if (r > rcut) continue;
                const double *t = tab + 7 * (types[i] * ntyp + types[j]);
                double a = t[0], b = t[1], c = t[2], dd = t[3], s = t[4], al = t[5], be = t[6];
                double fm = b * a * exp(b * (s - r)) - 6 * c / pow(r, 7) - 8 * dd / pow(r, 9) - al;
                double vm = a * exp(b * (s - r)) - c / pow(r, 6) - dd / pow(r, 8) + al * r + be;
                fx += fm * (d[0] / r);
                fy += fm * (d[1] / r);
                fz += fm * (d[2] / r);
                erow[ne++] = vm;
            }
            ecnt[i - i0] = ne;
            f[3 * i] = fx; f[3 * i + 1] = fy; f[3 * i + 2] = fz;
        }
        for (long i = i0; i < i1; i++) {
            const double *erow = ebuf + (i - i0) * np;
            for (long e = 0; e < ecnt[i - i0]; e++) en += erow[e];
        }
    }
    free(ebuf); free(ecnt);
    return en / 2;
}

/* Lennard-Jones table per type pair [sigma, epsilon, alpha, beta, 0, 0, 0] with the
   shifted-force constants at r_cut = L/2 (particles.c:230-266). pot_params holds
   [sigma, epsilon] per type pair, the layout solver.py:241-270 passes; the reference
   indexes it with a stride of 4 (particles.c:241), which reads past the array for two
   or more types -- with one type both agree. */
void orc_lj_table(const double *pp, int ntyp, double L, double *tab) {
    double rc = L / 2.0;
    for (int t = 0; t < ntyp * ntyp; t++) {
        double sigma = pp[2 * t], eps = pp[2 * t + 1];
        double vs = 4 * eps * (pow(sigma / rc, 12) - pow(sigma / rc, 6));
        double al = 4 * (12 * eps * pow(sigma / rc, 12) - 6 * eps * pow(sigma / rc, 6)) / rc;
        double be = -vs - al * rc;
        double *o = tab + 7 * t;
        o[0] = sigma; o[1] = eps; o[2] = al; o[3] = be; o[4] = 0; o[5] = 0; o[6] = 0;
    }
}

/* All-pairs shifted-force Lennard-Jones, both orders, j ascending (forces.c:199-271).
   Returns half the summed pair energy. */
double orc_lj_forces(const double *pos, const int32_t *types, const double *tab, int ntyp, int np,
                     double L, double rcut, double *f) {
    double en = 0.0;
    for (long i = 0; i < np; i++) {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (long j = 0; j < np; j++) {
            if (i == j) continue;
            double d[3], r;
            double x = pos[3 * i] - pos[3 * j];
            x -= L * round(x / L);
            r = x * x;
            d[0] = x;
            x = pos[3 * i + 1] - pos[3 * j + 1];
            x -= L * round(x / L);
            d[1] = x;
            r += x * x;
            x = pos[3 * i + 2] - pos[3 * j + 2];
            x -= L * round(x / L);
            d[2] = x;
            r += x * x;
            r = sqrt(r);
            if (r > rcut) continue;
            d[0] /= r; d[1] /= r; d[2] /= r;
            const double *t = tab + 7 * (types[i] * ntyp + types[j]);
            double sigma = t[0], eps = t[1], al = t[2], be = t[3];
            double fm = 4 * eps * (12 * pow(sigma / r, 12) - 6 * pow(sigma / r, 6)) / r - al;
            double vm = 4 * eps * (pow(sigma / r, 12) - pow(sigma / r, 6)) + al * r + be;
            fx += fm * d[0];
            fy += fm * d[1];
            fz += fm * d[2];
            en += vm;
        }
        f[3 * i] = fx; f[3 * i + 1] = fy; f[3 * i + 2] = fz;
    }
    return en / 2;
}

/* Soft-core repulsion table [nu, d, B, alpha, beta, 0, 0] (particles.c:268-295; the same
   for every type pair). */
void orc_sc_table(const double *pp, int ntyp, double L, double *tab) {
    double nu = pp[0], d = pp[1], B = pp[2], rc = 0.5 * L;
    double dr = d / rc, drp = pow(dr, nu);
    double al = B * nu * drp / rc;
    double be = -B * drp - al * rc;
    for (int t = 0; t < ntyp * ntyp; t++) {
        double *o = tab + 7 * t;
        o[0] = nu; o[1] = d; o[2] = B; o[3] = al; o[4] = be; o[5] = 0; o[6] = 0;
    }
}

/* Soft-core forces over pairs i < j with Newton's third law (forces.c:283-337), serial
   semantics: the reference's `omp parallel` without `for` runs the whole loop on every
   thread, which multiplies forces and energy by the thread count above one thread.
   Returns the summed pair energy. */
double orc_sc_forces(const double *pos, const double *tab, int np, double L, double rcut, double *f) {
    double nu = tab[0], d = tab[1], B = tab[2], al = tab[3], be = tab[4], en = 0.0;
    memset(f, 0, (size_t)3 * np * sizeof(double));
    for (long i = 0; i < np; i++) {
        for (long j = i + 1; j < np; j++) {
            double rd[3], r = 0.0;
            for (int k = 0; k < 3; k++) {
                double x = pos[3 * i + k] - pos[3 * j + k];
                x -= L * round(x / L);
                r += x * x;
                rd[k] = x;
            }
            r = sqrt(r);
            if (r > rcut) continue;
            double p = pow(d / r, nu);
            double vm = B * p + al * r + be;
            double fm = B * nu * p / r - al;
            for (int k = 0; k < 3; k++) {
                double fk = fm * rd[k] / r;
                f[3 * i + k] += fk;
                f[3 * j + k] -= fk;
            }
            en += vm;
        }
    }
    return en;
}

/* Linked cells as a CSR list: cell (IX,IY,IZ) with IX = int((nc/L) * x)
   (maze_poisson/linkedcell.py:18-26), ions of a cell in ascending index (the reverse of
   the reference's header/link chain). Out-of-range coordinates are clamped. */
void orc_cell_list(const double *pos, int np, double L, int nc, int32_t *start, int32_t *ions) {
    long ncell = (long)nc * nc * nc;
    double rel = nc / L;
    int32_t *cell = malloc((size_t)(np > 0 ? np : 1) * sizeof(int32_t));
    memset(start, 0, (ncell + 1) * sizeof(int32_t));
    for (long p = 0; p < np; p++) {
        long c[3];
        for (int d = 0; d < 3; d++) {
            long v = (long)(rel * pos[3 * p + d]);
            c[d] = v < 0 ? 0 : (v >= nc ? nc - 1 : v);
        }
        cell[p] = (int32_t)((c[0] * nc + c[1]) * nc + c[2]);
        start[cell[p] + 1]++;
    }
    for (long c = 0; c < ncell; c++) start[c + 1] += start[c];
    int32_t *fill = malloc((size_t)ncell * sizeof(int32_t));
    memcpy(fill, start, ncell * sizeof(int32_t));
    for (long p = 0; p < np; p++) ions[fill[cell[p]]++] = (int32_t)p;
    free(fill); free(cell);
}

/* ------------------------------------------------------------------------------------
 * Facade (library/src/solver_md.c) over one global system.
 * ---------------------------------------------------------------------------------- */
enum { G_LCG = 0, G_FFT = 1, G_MG = 2, G_MAZE_LCG = 3, G_MAZE_MG = 4 };
enum { P_NONE = 0, P_JACOBI = 1, P_MG = 2, P_SSOR = 3, P_BLOCKJACOBI = 4 };

static struct {
    int type, precond, n;
    double L, h, tol, eps_s, eps_int;
    long m;
    double *q, *phi, *phi_prev, *y;
    int pb, nonpolar;                    /* grid_general.c:84-100 */
    double w, kbar2;
    double *ex, *ey, *ez, *k2;
} G;
static struct {
    int np, ntyp, n;
    double L, h, rcut;
    int32_t *types;
    double *pos, *vel, *fe, *fn, *ft, *mass, *chg, *tab;
    int64_t *nbr;
    int cas, nnb, pot;
    int pb;                              /* particles.c:111-127 */
    double gamma_np, beta_np;
    double *radii, *fdb, *fib, *fnp;
} P;
static struct {
    int type, enabled;
    double dt, T, c1, c2;
} I;
static double q_tot_prev = 0.0; /* persists across systems, solver_md.c:16 */
static double *noise = NULL;
static long noise_len = 0, noise_pos = 0;

static void die(const char *msg) { fprintf(stderr, "oracle: %s\n", msg); exit(1); }

void solver_initialize(void) {}

void solver_initialize_grid(int n, double L, double h, double tol, double eps_s, double eps_int,
                            int grid_type, int precond_type) {
    if (grid_type == G_FFT) die("FFT is restated in numpy (oracle/fft_oracle.py)");
    if (grid_type < 0 || grid_type > 4) die("bad grid type");
    if (precond_type < 0 || precond_type > P_BLOCKJACOBI) die("bad preconditioner type");
    G.type = grid_type; G.precond = precond_type; G.n = n;
    G.L = L; G.h = h; G.tol = tol; G.eps_s = eps_s; G.eps_int = eps_int;
    G.m = (long)n * n * n;
    G.pb = 0; G.nonpolar = 0;
    G.q = calloc(G.m, sizeof(double)); G.phi = calloc(G.m, sizeof(double));
    G.phi_prev = calloc(G.m, sizeof(double)); G.y = calloc(G.m, sizeof(double));
}

void solver_initialize_particles(int n, int n_typ, double L, double h, int n_p, int pot_type,
                                 int cas_type, int *types, double *pos, double *vel, double *mass,
                                 double *charges, double *pot_params) {
    if (pot_type < 0 || pot_type > 2) die("bad potential type");
    if (cas_type < 0 || cas_type > 2) die("bad charge assignment scheme");
    P.np = n_p; P.ntyp = n_typ; P.n = n; P.L = L; P.h = h; P.rcut = L / 2.0;
    P.cas = cas_type; P.nnb = scheme_points(cas_type);
    size_t v3 = (size_t)3 * n_p * sizeof(double);
    P.types = malloc(n_p * sizeof(int32_t)); memcpy(P.types, types, n_p * sizeof(int32_t));
    P.pos = malloc(v3); memcpy(P.pos, pos, v3);
    P.vel = malloc(v3); memcpy(P.vel, vel, v3);
    P.mass = malloc(n_p * sizeof(double)); memcpy(P.mass, mass, n_p * sizeof(double));
    P.chg = malloc(n_p * sizeof(double)); memcpy(P.chg, charges, n_p * sizeof(double));
    P.fe = calloc(3 * n_p, sizeof(double)); P.fn = calloc(3 * n_p, sizeof(double));
    P.ft = calloc(3 * n_p, sizeof(double));
    P.nbr = malloc((size_t)n_p * P.nnb * 3 * sizeof(int64_t));
    P.tab = malloc((size_t)n_typ * n_typ * 7 * sizeof(double));
    P.pot = pot_type;
    P.pb = 0;
    if (pot_type == 0) orc_tf_table(pot_params, n_typ, L, P.tab);
    else if (pot_type == 1) orc_lj_table(pot_params, n_typ, L, P.tab);
    else orc_sc_table(pot_params, n_typ, L, P.tab);
}

void solver_initialize_integrator(int n_p, double dt, double T, double gamma, int itg_type,
                                  int itg_enabled) {
    (void)n_p;
    I.type = itg_type; I.dt = dt; I.enabled = 0; I.c1 = 1.0; I.c2 = 1.0; I.T = 0.0;
    if (itg_enabled == 1) {                 /* integrator_{ovrvo,verlet}.c init_thermostat */
        I.T = T; I.enabled = 1;
        if (itg_type == 0) {
            I.c1 = exp(-gamma * dt);
            I.c2 = sqrt(2 / (gamma * dt) * tanh(0.5 * gamma * dt));
        }
    }
}

int solver_update_charges(void) {
    if (P.cas == 0) orc_cic_neighbors(P.pos, P.np, P.n, P.h, P.nbr);
    else orc_spline_neighbors(P.pos, P.np, P.n, P.h, P.nbr);
    double qt = spread_scheme(P.pos, P.chg, P.nbr, P.nnb, P.np, G.n, G.h, G.q, scheme_weight(P.cas));
    if (fabs(q_tot_prev - qt) > 1e-6) {
        printf("Charge conservation error: q_tot = %.6f, q_tot_loc = %.6f\n", q_tot_prev, qt);
        exit(1);
    }
    q_tot_prev = qt;
    return 0;
}

/* -4 pi / h, divided by eps_s unless PB carries the dielectric in the operator
   (grid_lcg.c:100-110) */
static double rhs_const(void) {
    double c = -4 * PI_D / G.h;
    if (!G.pb) c /= G.eps_s;
    return c;
}
static void lap_pb(const double *u, double *out) { orc_laplace_pb(u, out, G.ex, G.ey, G.ez, G.k2, G.n); }

/* grid_lcg.c:100-124, grid_maze_lcg.c:107-126, grid_multigrid.c:86-108,
   grid_maze_multigrid.c:86-112: all four solve L phi = -4 pi q/(h eps) by CG from 0. */
void solver_init_field(void) {
    double c = rhs_const();
    memset(G.y, 0, G.m * sizeof(double));
    memcpy(G.phi_prev, G.phi, G.m * sizeof(double));
    scaled_copy(G.phi, G.q, c, G.m);
    if (G.pb) orc_conj_grad_pb(G.phi, G.y, G.phi, G.tol, G.n, G.ex, G.ey, G.ez, G.k2);
    else orc_conj_grad(G.phi, G.y, G.phi, G.tol, G.n);
}

/* phi <- 2 phi - phi_prev, phi_prev <- old phi (verlet.c:46-51, grid_multigrid.c:124-129) */
static void extrapolate(void) {
#pragma omp parallel for num_threads(orc_threads()) if (G.m >= PAR_MIN)
    for (long t = 0; t < G.m; t++) {
        double a = G.phi[t];
        G.phi[t] = 2 * a - G.phi_prev[t];
        G.phi_prev[t] = a;
    }
}

int solver_update_field(void) {
    long m = G.m;
    int n = G.n, res = -1;
    if (G.type == G_LCG) {                                 /* grid_lcg.c:126-149 */
        double c = rhs_const();
        memcpy(G.phi_prev, G.phi, m * sizeof(double));
        scaled_copy(G.y, G.q, c, m);
        if (G.pb) return orc_conj_grad_pb(G.y, G.phi_prev, G.phi, G.tol, n, G.ex, G.ey, G.ez, G.k2);
        return orc_conj_grad(G.y, G.phi_prev, G.phi, G.tol, n);
    }
    if (G.pb && G.type == G_MAZE_LCG) {                    /* verlet.c:152-193 */
        double *tmp = malloc(m * sizeof(double));
        extrapolate();
        lap_pb(G.phi, tmp);
        axpy(tmp, G.q, (4 * PI_D) / G.h, m);
        res = orc_conj_grad_pb(tmp, G.y, G.y, G.tol, n, G.ex, G.ey, G.ez, G.k2);
        axpy(G.phi, G.y, -1.0, m);
        free(tmp);
        return res;
    }
    if (G.pb) {                                            /* grid_multigrid.c:151-177, verlet.c:212-271 */
        double *tmp = malloc(m * sizeof(double)), *tmp2 = malloc(m * sizeof(double));
        int it = 0;
        extrapolate();
        if (G.type == G_MG) {
            double c = rhs_const();
            scaled_copy(tmp, G.q, c, m);
            while (it < 1000) {
                orc_mg_pb_apply(tmp, G.phi, n, 4, G.ex, G.ey, G.ez, G.k2);
                lap_pb(G.phi, tmp2);
                axpy(tmp2, tmp, -1.0, m);
                double a = amax(tmp2, m);
                it++;
                if (a <= G.tol) { res = it; break; }
            }
        } else {
            lap_pb(G.phi, tmp2);
            axpy(tmp2, G.q, (4 * PI_D) / G.h, m);
            while (it < 1000) {
                orc_mg_pb_apply(tmp2, G.y, n, 4, G.ex, G.ey, G.ez, G.k2);
                lap_pb(G.y, tmp);
                axpy(tmp, tmp2, -1., m);
                double a = amax(tmp, m);
                it++;
                if (a <= G.tol) { res = it; break; }
            }
            axpy(G.phi, G.y, -1.0, m);
            if (G.precond != P_NONE) die("Maze Multigrid with preconditioner not implemented");
        }
        free(tmp); free(tmp2);
        return res;
    }
    if (G.type == G_MAZE_LCG) {                            /* verlet.c:31-71 */
        double hh = G.h * G.eps_s;
        double *tmp = malloc(m * sizeof(double));
        extrapolate();
        orc_laplace(G.phi, tmp, n);
        axpy(tmp, G.q, (4 * PI_D) / hh, m);
        if (G.precond == P_NONE) res = orc_conj_grad(tmp, G.y, G.y, G.tol, n);
        else res = conj_grad_precond(tmp, G.y, G.y, G.tol, n, G.precond);
        axpy(G.phi, G.y, -1.0, m);
        free(tmp);
        return res;
    }
    double *tmp = malloc(m * sizeof(double)), *tmp2 = malloc(m * sizeof(double));
    int it = 0;
    if (G.type == G_MG) {                                  /* grid_multigrid.c:110-212 */
        extrapolate();
        double c = rhs_const();
        scaled_copy(tmp, G.q, c, m);
        while (it < 1000) {
            orc_mg_apply(tmp, G.phi, n, 3);
            orc_laplace(G.phi, tmp2, n);
            axpy(tmp2, tmp, -1.0, m);
            double a = amax(tmp2, m);
            it++;
            if (a <= G.tol) { res = it; break; }
        }
    } else {                                               /* verlet.c:86-149 */
        double hh = G.h * G.eps_s;
        extrapolate();
        orc_laplace(G.phi, tmp2, n);
        axpy(tmp2, G.q, (4 * PI_D) / hh, m);
        while (it < 1000) {
            orc_mg_apply(tmp2, G.y, n, 3);
            orc_laplace(G.y, tmp, n);
            axpy(tmp, tmp2, -1., m);
            double a = amax(tmp, m);
            it++;
            if (a <= G.tol) { res = it; break; }
        }
        axpy(G.phi, G.y, -1.0, m);
        if (G.precond != P_NONE) die("Maze Multigrid with preconditioner not implemented");
    }
    free(tmp); free(tmp2);
    return res;
}

void solver_set_field(double *phi) { memcpy(G.phi, phi, G.m * sizeof(double)); }
void solver_set_field_prev(double *phi) { memcpy(G.phi_prev, phi, G.m * sizeof(double)); }

void solver_compute_forces_elec(void) {
    force_scheme(G.phi, P.nbr, P.nnb, P.chg, P.pos, P.np, P.n, P.h, P.fe, scheme_weight(P.cas));
}
double solver_compute_forces_noel(void) {
    if (P.pot == 1) return orc_lj_forces(P.pos, P.types, P.tab, P.ntyp, P.np, P.L, P.rcut, P.fn);
    if (P.pot == 2) return orc_sc_forces(P.pos, P.tab, P.np, P.L, P.rcut, P.fn);
    return orc_tf_forces(P.pos, P.types, P.tab, P.ntyp, P.np, P.L, P.rcut, P.fn);
}
void solver_compute_forces_tot(void) {                     /* particles.c:777-795 */
    for (long t = 0; t < 3L * P.np; t++) {
        double v = 0.0;
        v += 1.0 * P.fe[t];
        v += 1.0 * P.fn[t];
        if (P.pb) { v += 1.0 * P.fdb[t]; v += 1.0 * P.fib[t]; v += 1.0 * P.fnp[t]; }
        P.ft[t] = v;
    }
}

double get_kinetic_energy(void) {                          /* particles.c:802-820 */
    double kin = 0.0;
    for (long p = 0; p < P.np; p++) {
        double a = 0.0;
        for (int d = 0; d < 3; d++) a += pow(P.vel[3 * p + d], 2);
        kin += P.mass[p] * a;
    }
    return 0.5 * kin;
}
double get_temperature(void) { return 2 * get_kinetic_energy() / (3 * P.np * KB_HARTREE); }

static double next_noise(void) {
    if (noise_pos >= noise_len) die("injected noise exhausted");
    return noise[noise_pos++];
}
void orc_set_noise(const double *z, int64_t count) {
    free(noise);
    noise = malloc((size_t)(count > 0 ? count : 1) * sizeof(double));
    memcpy(noise, z, (size_t)count * sizeof(double));
    noise_len = count; noise_pos = 0;
}

static inline double wrap_box(double a, double L) {
    if (a < 0) return a + L;
    if (a >= L) return a - L;
    return a;
}

/* integrator_ovrvo.c:45-78 with injected N(0,1) draws */
static void o_block(void) {
    double c1s = sqrt(I.c1), var2 = (1 - I.c1) * KB_HARTREE * I.T;
    for (long p = 0; p < P.np; p++) {
        double var1 = sqrt(var2 / P.mass[p]);
        for (int d = 0; d < 3; d++) {
            P.vel[3 * p + d] *= c1s;
            P.vel[3 * p + d] += var1 * next_noise();
        }
    }
}
static void v_block(void) {                                /* integrator_ovrvo.c:80-96 */
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++)
            P.vel[3 * p + d] += 0.5 * I.dt * I.c2 * P.ft[3 * p + d] / P.mass[p];
}
static void r_block(void) {                                /* integrator_ovrvo.c:98-123 */
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++)
            P.pos[3 * p + d] = wrap_box(P.pos[3 * p + d] + I.c2 * I.dt * P.vel[3 * p + d], P.L);
}

void integrator_part_1(void) {
    if (I.type == 0) {                                     /* integrator_ovrvo.c:125-131 */
        if (I.enabled) o_block();
        v_block();
        r_block();
        return;
    }
    if (I.enabled) {                                       /* integrator_verlet.c:12-53 */
        double s = sqrt(I.T / get_temperature());
        for (long t = 0; t < 3L * P.np; t++) P.vel[t] *= s;
    }
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++) {
            long t = 3 * p + d;
            P.vel[t] += 0.5 * I.dt * P.ft[t] / P.mass[p];
            P.pos[t] = wrap_box(P.pos[t] + I.dt * P.vel[t], P.L);
        }
}

void integrator_part_2(void) {
    if (I.type == 0) {
        v_block();
        if (I.enabled) o_block();
        return;
    }
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++)
            P.vel[3 * p + d] += 0.5 * I.dt * P.ft[3 * p + d] / P.mass[p];
}

int solver_check_thermostat(void) {                        /* solver_md.c:210-221 */
    if (I.enabled == 1 && fabs(get_temperature() - I.T) < 100) {
        I.enabled = 0;
        if (I.type == 0) { I.c1 = 1.0; I.c2 = 1.0; }
        return 1;
    }
    return 0;
}

void solver_rescale_velocities(void) {                     /* particles.c:841-857 */
    double *iv = calloc((size_t)P.ntyp * 3, sizeof(double));
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++) iv[P.types[p] * 3 + d] += P.vel[3 * p + d];
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++) P.vel[3 * p + d] -= 2 * iv[P.types[p] * 3 + d] / P.np;
    free(iv);
}

void solver_finalize(void) {
    free(G.q); free(G.phi); free(G.phi_prev); free(G.y);
    free(P.types); free(P.pos); free(P.vel); free(P.mass); free(P.chg);
    free(P.fe); free(P.fn); free(P.ft); free(P.nbr); free(P.tab);
    free(G.ex); free(G.ey); free(G.ez); free(G.k2);
    free(P.radii); free(P.fdb); free(P.fib); free(P.fnp);
    memset(&G, 0, sizeof(G)); memset(&P, 0, sizeof(P));
}

void get_pos(double *o) { memcpy(o, P.pos, 3 * (size_t)P.np * sizeof(double)); }
void get_vel(double *o) { memcpy(o, P.vel, 3 * (size_t)P.np * sizeof(double)); }
void get_fcs_elec(double *o) { memcpy(o, P.fe, 3 * (size_t)P.np * sizeof(double)); }
void get_fcs_noel(double *o) { memcpy(o, P.fn, 3 * (size_t)P.np * sizeof(double)); }
void get_fcs_tot(double *o) { memcpy(o, P.ft, 3 * (size_t)P.np * sizeof(double)); }
void get_field(double *o) { memcpy(o, G.phi, G.m * sizeof(double)); }
void get_field_prev(double *o) { memcpy(o, G.phi_prev, G.m * sizeof(double)); }
void get_q(double *o) { memcpy(o, G.q, G.m * sizeof(double)); }
void get_momentum(double *o) {                             /* particles.c:822-839 */
    double s[3] = {0.0, 0.0, 0.0};
    for (long p = 0; p < P.np; p++)
        for (int d = 0; d < 3; d++) s[d] += P.mass[p] * P.vel[3 * p + d];
    o[0] = s[0]; o[1] = s[1]; o[2] = s[2];
}

/* ---- remaining facade symbols (enum tables, serial MPI stubs, trivial getters) ---- */
static char grid_names[5][16] = {"LCG", "FFT", "MULTIGRID", "MAZE-LCG", "MAZE-MULTIGRID"};
static char precond_names[5][16] = {"NONE", "JACOBI", "MG", "SSOR", "BLOCKJACOBI"};
static char pot_names[3][16] = {"TF", "LJ", "SC"};
static char cas_names[3][16] = {"CIC", "SPL_QUADR", "SPL_CUBIC"};
static char itg_names[2][16] = {"OVRVO", "VERLET"};
int init_mpi(void) { return 0; }
int get_rank(void) { return 0; }
int get_grid_type_num(void) { return 5; }
char *get_grid_type_str(int i) { return grid_names[i]; }
int get_precond_type_num(void) { return 5; }
char *get_precond_type_str(int i) { return precond_names[i]; }
int get_potential_type_num(void) { return 3; }
char *get_potential_type_str(int i) { return pot_names[i]; }
int get_ca_scheme_type_num(void) { return 3; }
char *get_ca_scheme_type_str(int i) { return cas_names[i]; }
int get_integrator_type_num(void) { return 2; }
char *get_integrator_type_str(int i) { return itg_names[i]; }
void solver_initialize_grid_pois_boltz(double w, double kbar2, int nonpolar) {  /* grid_general.c:84-100 */
    G.pb = 1; G.nonpolar = nonpolar; G.w = w; G.kbar2 = kbar2;
    G.ex = calloc(G.m, sizeof(double)); G.ey = calloc(G.m, sizeof(double));
    G.ez = calloc(G.m, sizeof(double)); G.k2 = calloc(G.m, sizeof(double));
}
void solver_initialize_particles_pois_boltz(double gamma_np, double beta_np, double *radii) {
    P.pb = 1; P.gamma_np = gamma_np; P.beta_np = beta_np;   /* particles.c:111-127 */
    P.radii = malloc((size_t)P.np * sizeof(double));
    memcpy(P.radii, radii, (size_t)P.np * sizeof(double));
    P.fdb = calloc(3 * (size_t)P.np, sizeof(double)); P.fib = calloc(3 * (size_t)P.np, sizeof(double));
    P.fnp = calloc(3 * (size_t)P.np, sizeof(double));
}
void solver_update_eps_k2(void) {                           /* solver_md.c:131-133 */
    orc_update_eps_k2(P.pos, P.radii, P.np, G.n, G.h, G.w, G.eps_s, G.eps_int, G.kbar2, G.ex, G.ey,
                      G.ez, G.k2);
}
double solver_compute_forces_pb(void) {                     /* particles.c:420-775 */
    if (!G.pb) die("Poisson-Boltzmann forces are not enabled in the grid.");
    orc_forces_pb(P.pos, P.radii, P.np, G.n, G.h, G.w, G.eps_s, G.eps_int, P.gamma_np, G.nonpolar, G.phi,
                  G.ex, G.ey, G.ez, G.k2, P.fdb, P.fib, P.fnp);
    return 0.0;  /* the reference's non_polar_energy is never accumulated */
}
void get_fcs_db(double *o) {
    if (P.pb) memcpy(o, P.fdb, 3 * (size_t)P.np * sizeof(double));
    else memset(o, 0, 3 * (size_t)P.np * sizeof(double));
}
void get_fcs_ib(double *o) {
    if (P.pb) memcpy(o, P.fib, 3 * (size_t)P.np * sizeof(double));
    else memset(o, 0, 3 * (size_t)P.np * sizeof(double));
}
void get_fcs_np(double *o) {
    if (P.pb) memcpy(o, P.fnp, 3 * (size_t)P.np * sizeof(double));
    else memset(o, 0, 3 * (size_t)P.np * sizeof(double));
}
/* the PB face / cell coefficients of the current grid (no reference getter) */
void orc_get_pb_grids(double *ex, double *ey, double *ez, double *k2) {
    size_t b = G.m * sizeof(double);
    memcpy(ex, G.ex, b); memcpy(ey, G.ey, b); memcpy(ez, G.ez, b); memcpy(k2, G.k2, b);
}
void get_charges(double *o) { memcpy(o, P.chg, (size_t)P.np * sizeof(double)); }
void get_masses(double *o) { memcpy(o, P.mass, (size_t)P.np * sizeof(double)); }
void get_types(int *o) { memcpy(o, P.types, (size_t)P.np * sizeof(int32_t)); }
void get_radii(double *o) {
    if (P.pb) memcpy(o, P.radii, (size_t)P.np * sizeof(double));
    else memset(o, 0, (size_t)P.np * sizeof(double));
}
double get_energy_elec(void) {                             /* grid_general.c:304-315 */
    double e = 0.0;
    for (long t = 0; t < G.m; t++) e += 0.5 * G.phi[t];
    return e;
}
