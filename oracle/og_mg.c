/*
 * og_mg.c -- oracle (test infrastructure only): pressure projection of the
 * reference restated in FP64: SetPressureBC + SetupPoisson + checks
 * (modules.f90:916-949,2722-2892; newsolver.f90:275-344), the geometric
 * multigrid (MGsolver.f90:34-405, newsolver.f90:34-76,192-247),
 * project_velocity (paris.f90:882-909), calcResidual (modules.f90:3313-3387),
 * Setup_testMG (modules.f90:3160-3192) and get_MGtest_err (MGsolver.f90:407).
 *
 * The matrix A is stored as the reference stores A(is:ie,js:je,ks:ke,8):
 * component-major, A[c*N + (i + nx*(j + ny*k))], interior only.
 */
#include <math.h>
#include <stdio.h>
#include <omp.h>
#include <string.h>
#include "og.h"

/* mask of a face for the pressure equation: SetPressureBC zeroes the masks of
 * wall faces (bdry_cond 0 or 2), modules.f90:916-949.  dir 0..2, face index f
 * is the C ghosted index of u(f) (face f+1/2). */
static double og_mask(const og_grid* g, int dir, int f) {
    int lo = g->ng - 1, hi = g->ng + g->N[dir] - 1;   /* is-1 and ie */
    int bl = g->d.bdry_cond[dir], bh = g->d.bdry_cond[dir + 3];
    if (f == lo && (bl == 0 || bl == 2)) return 0.0;
    if (f == hi && (bh == 0 || bh == 2)) return 0.0;
    return 1.0;
}

/* SetupPoisson (modules.f90:2722-2753) with Poisson_BCs for walls/periodic
 * (no rows change for bdry_cond 0,1,2) and check_and_debug_Poisson +
 * check_poisson_setup (modules.f90:2894-2959; newsolver.f90:275-344).
 * Returns 0, or PARIS_SETUP_ERROR when a check of the reference fails. */
int og_setup_poisson(const paris_grid_desc* desc, const double* u, const double* v,
                     const double* w, const double* rho, double dt, double volsrc, double* A) {
    og_grid* g = og_grid_new(desc);
    int ng = g->ng, nx = g->nx, ny = g->ny, nz = g->nz;
    long N = (long)nx * ny * nz;
    long sy = g->sy, sz = g->sz;
    int status = 0;
#pragma omp parallel for schedule(static)
    for (int k = ng; k < ng + nz; k++)
        for (int j = ng; j < ng + ny; j++)
            for (int i = ng; i < ng + nx; i++) {
                long n = OG_IX(g, i, j, k);
                long m = (i - ng) + (long)nx * ((j - ng) + (long)ny * (k - ng));
                double a1 = 2.0 * dt * og_mask(g, 0, i - 1) / (g->dx[i] * g->dxh[i - 1] * (rho[n - 1] + rho[n]));
                double a2 = 2.0 * dt * og_mask(g, 0, i) / (g->dx[i] * g->dxh[i] * (rho[n + 1] + rho[n]));
                double a3 = 2.0 * dt * og_mask(g, 1, j - 1) / (g->dy[j] * g->dyh[j - 1] * (rho[n - sy] + rho[n]));
                double a4 = 2.0 * dt * og_mask(g, 1, j) / (g->dy[j] * g->dyh[j] * (rho[n + sy] + rho[n]));
                double a5 = 2.0 * dt * og_mask(g, 2, k - 1) / (g->dz[k] * g->dzh[k - 1] * (rho[n - sz] + rho[n]));
                double a6 = 2.0 * dt * og_mask(g, 2, k) / (g->dz[k] * g->dzh[k] * (rho[n + sz] + rho[n]));
                A[0 * N + m] = a1; A[1 * N + m] = a2; A[2 * N + m] = a3;
                A[3 * N + m] = a4; A[4 * N + m] = a5; A[5 * N + m] = a6;
                A[6 * N + m] = a1 + a2 + a3 + a4 + a5 + a6;
                A[7 * N + m] = -(volsrc + (u[n] - u[n - 1]) / g->dx[i] + (v[n] - v[n - sy]) / g->dy[j] +
                                 (w[n] - w[n - sz]) / g->dz[k]);
            }
    /* check_and_debug_Poisson: A7 < 1e-50 is only legal in a solid (all six
     * masks zero); then A8 must be ~0, A1..6 zero and A7 is set to 1. */
    for (int k = ng; k < ng + nz && !status; k++)
        for (int j = ng; j < ng + ny && !status; j++)
            for (int i = ng; i < ng + nx; i++) {
                long m = (i - ng) + (long)nx * ((j - ng) + (long)ny * (k - ng));
                if (A[6 * N + m] < 1e-50) {
                    int solid = og_mask(g, 0, i - 1) < 0.5 && og_mask(g, 0, i) < 0.5 && og_mask(g, 1, j - 1) < 0.5 &&
                                og_mask(g, 1, j) < 0.5 && og_mask(g, 2, k - 1) < 0.5 && og_mask(g, 2, k) < 0.5;
                    if (!solid || A[7 * N + m] > 1e-50) { status = PARIS_SETUP_ERROR; break; }
                    A[6 * N + m] = 1.0;
                }
            }
    /* check_poisson_setup: NaN / A7 < 1e-55, volume source, constant in kernel */
    if (!status) {
        double intsource = 0.0;
        for (long m = 0; m < N; m++) {
            for (int c = 0; c < 8; c++)
                if (A[c * N + m] != A[c * N + m]) status = PARIS_SETUP_ERROR;
            if (A[6 * N + m] < 1e-55) status = PARIS_SETUP_ERROR;
        }
        for (long m = 0; m < N; m++) intsource += A[7 * N + m];
        if (intsource / (double)N > 1e-10) status = PARIS_SETUP_ERROR;
        for (int k = ng; k < ng + nz && !status; k++)
            for (int j = ng; j < ng + ny && !status; j++)
                for (int i = ng; i < ng + nx; i++) {
                    long m = (i - ng) + (long)nx * ((j - ng) + (long)ny * (k - ng));
                    double a7 = A[6 * N + m];
                    if (og_mask(g, 0, i - 1) < 0.5 && og_mask(g, 0, i) < 0.5 && og_mask(g, 1, j - 1) < 0.5 &&
                        og_mask(g, 1, j) < 0.5 && og_mask(g, 2, k - 1) < 0.5 && og_mask(g, 2, k) < 0.5)
                        a7 = 0.0;
                    double s = A[0 * N + m] + A[1 * N + m] + A[2 * N + m] + A[3 * N + m] + A[4 * N + m] + A[5 * N + m];
                    if (fabs(s - a7) > 1e-10) { status = PARIS_SETUP_ERROR; break; }
                }
    }
    og_grid_free(g);
    return status;
}

/* Setup_testMG (modules.f90:3160-3192); pi is the single-precision literal
 * 3.14159265359 held in real(8). */
int og_setup_testmg(const paris_grid_desc* desc, const double* rho, double* A) {
    og_grid* g = og_grid_new(desc);
    const double pi = (double)3.14159265359f;
    int ng = g->ng, nx = g->nx, ny = g->ny, nz = g->nz;
    long N = (long)nx * ny * nz, sy = g->sy, sz = g->sz;
    for (int k = ng; k < ng + nz; k++)
        for (int j = ng; j < ng + ny; j++)
            for (int i = ng; i < ng + nx; i++) {
                long n = OG_IX(g, i, j, k);
                long m = (i - ng) + (long)nx * ((j - ng) + (long)ny * (k - ng));
                double a1 = 2.0 / (g->dx[i] * g->dxh[i - 1] * (rho[n - 1] + rho[n]));
                double a2 = 2.0 / (g->dx[i] * g->dxh[i] * (rho[n + 1] + rho[n]));
                double a3 = 2.0 / (g->dy[j] * g->dyh[j - 1] * (rho[n - sy] + rho[n]));
                double a4 = 2.0 / (g->dy[j] * g->dyh[j] * (rho[n + sy] + rho[n]));
                double a5 = 2.0 / (g->dz[k] * g->dzh[k - 1] * (rho[n - sz] + rho[n]));
                double a6 = 2.0 / (g->dz[k] * g->dzh[k] * (rho[n + sz] + rho[n]));
                A[0 * N + m] = a1; A[1 * N + m] = a2; A[2 * N + m] = a3;
                A[3 * N + m] = a4; A[4 * N + m] = a5; A[5 * N + m] = a6;
                A[6 * N + m] = a1 + a2 + a3 + a4 + a5 + a6;
                A[7 * N + m] = 3.0 * ((2.0 * pi) * (2.0 * pi)) * sin(2. * pi * g->x[i]) * sin(2. * pi * g->y[j]) *
                               sin(2. * pi * g->z[k]);
            }
    og_grid_free(g);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Multigrid hierarchy: level L (1..LMG) has n_L = nd/2^(LMG-L) cells; K holds
 * the 8 components without ghosts, p and e have one... Ng ghost layers.     */
typedef struct {
    int n[3];
    long N;            /* interior cells */
    int nt[3];         /* with ghosts */
    long sy, sz, ntot;
    double* K;         /* 8*N */
    double* p;         /* pMG */
    double* e;         /* EMG */
} og_level;

typedef struct {
    og_grid* g;
    int LMG;
    og_level* lev;     /* lev[1..LMG] */
    int nrelax, sym;
} og_mg;

#define LIX(l, i, j, k) ((long)(i) + (long)(j) * (l)->sy + (long)(k) * (l)->sz)

static og_mg* og_mg_new(og_grid* g) {
    og_mg* mg = calloc(1, sizeof(og_mg));
    mg->g = g;
    int Lmin = 1000;
    for (int a = 0; a < 3; a++) {
        int nd = g->N[a], L = 0;
        while ((1 << (L + 1)) <= nd) L++;
        if (L < Lmin) Lmin = L;
    }
    mg->LMG = Lmin;
    mg->lev = calloc(Lmin + 1, sizeof(og_level));
    for (int L = Lmin; L >= 1; L--) {
        og_level* l = &mg->lev[L];
        for (int a = 0; a < 3; a++) {
            l->n[a] = g->N[a] >> (Lmin - L);
            l->nt[a] = l->n[a] + 2 * g->ng;
        }
        l->N = (long)l->n[0] * l->n[1] * l->n[2];
        l->sy = l->nt[0];
        l->sz = (long)l->nt[0] * l->nt[1];
        l->ntot = l->sz * l->nt[2];
        l->K = calloc(8 * l->N, sizeof(double));
        l->p = calloc(l->ntot, sizeof(double));
        l->e = calloc(l->ntot, sizeof(double));
    }
    mg->nrelax = g->d.nrelax > 0 ? g->d.nrelax : 3;
    mg->sym = g->d.sym_mg;
    return mg;
}

static void og_mg_free(og_mg* mg) {
    for (int L = 1; L <= mg->LMG; L++) {
        free(mg->lev[L].K); free(mg->lev[L].p); free(mg->lev[L].e);
    }
    free(mg->lev);
    free(mg);
}

/* ghost_MG_x/y/z with one layer (apply_BC_MG, newsolver.f90:192-206) */
static void og_apply_bc_mg(const og_mg* mg, const og_level* l, double* F) {
    int ng = mg->g->ng;
    long st[3] = {1, l->sy, l->sz};
    for (int dir = 0; dir < 3; dir++) {
        if (!og_is_periodic(mg->g, dir)) continue;
        int lo = ng, hi = ng + l->n[dir] - 1;
        int o1 = (dir + 1) % 3, o2 = (dir + 2) % 3;
        for (int b = 0; b < l->nt[o2]; b++)
            for (int a = 0; a < l->nt[o1]; a++) {
                double* base = F + a * st[o1] + b * st[o2];
                base[(lo - 1) * st[dir]] = base[hi * st[dir]];
                base[(hi + 1) * st[dir]] = base[lo * st[dir]];
            }
    }
}

/* RedBlackRelax, newsolver.f90:209-247: pass 1 updates cells with
 * (i-is)+(j-js)+(k-ks) even, then the one-layer halo, then pass 2. */
static void og_rb_relax(const og_mg* mg, const og_level* l, const double* A, double* p, double beta) {
    int ng = mg->g->ng;
    long N = l->N;
    for (int pass = 0; pass < 2; pass++) {
#pragma omp parallel for schedule(static)
        for (int k = 0; k < l->n[2]; k++)
            for (int j = 0; j < l->n[1]; j++) {
                int i0 = (j + k + pass) & 1;
                for (int i = i0; i < l->n[0]; i += 2) {
                    long m = i + (long)l->n[0] * (j + (long)l->n[1] * k);
                    long q = LIX(l, i + ng, j + ng, k + ng);
                    p[q] = (1.0 - beta) * p[q] +
                           beta / A[6 * N + m] *
                               (A[0 * N + m] * p[q - 1] + A[1 * N + m] * p[q + 1] + A[2 * N + m] * p[q - l->sy] +
                                A[3 * N + m] * p[q + l->sy] + A[4 * N + m] * p[q - l->sz] +
                                A[5 * N + m] * p[q + l->sz] + A[7 * N + m]);
                }
            }
        if (pass == 0) og_apply_bc_mg(mg, l, p);
    }
}

/* get_residual, MGsolver.f90:84-104: A8 <- A8 - A7 p + sum A_n p_n, returns sum |A8|^norm */
static double og_get_residual(const og_mg* mg, const og_level* l, double* A, const double* p, int norm) {
    int ng = mg->g->ng;
    long N = l->N;
    double en = 0.0;
#pragma omp parallel for reduction(+ : en) schedule(static)
    for (int k = 0; k < l->n[2]; k++)
        for (int j = 0; j < l->n[1]; j++)
            for (int i = 0; i < l->n[0]; i++) {
                long m = i + (long)l->n[0] * (j + (long)l->n[1] * k);
                long q = LIX(l, i + ng, j + ng, k + ng);
                double r = A[7 * N + m] - A[6 * N + m] * p[q] + A[0 * N + m] * p[q - 1] + A[1 * N + m] * p[q + 1] +
                           A[2 * N + m] * p[q - l->sy] + A[3 * N + m] * p[q + l->sy] +
                           A[4 * N + m] * p[q - l->sz] + A[5 * N + m] * p[q + l->sz];
                A[7 * N + m] = r;
                double ar = fabs(r);
                en = en + (norm == 2 ? ar * ar : (norm == 1 ? ar : pow(ar, norm)));
            }
    return en;
}

/* compute_residual, MGsolver.f90:106-126 (A from the caller, p ghosted) */
static double og_compute_residual(const og_grid* g, const double* A, const double* p, int norm) {
    int ng = g->ng, nx = g->nx, ny = g->ny, nz = g->nz;
    long N = (long)nx * ny * nz;
    double en = 0.0;
#pragma omp parallel for reduction(+ : en) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long m = i + (long)nx * (j + (long)ny * k);
                long q = OG_IX(g, i + ng, j + ng, k + ng);
                double r = A[7 * N + m] - A[6 * N + m] * p[q] + A[0 * N + m] * p[q - 1] + A[1 * N + m] * p[q + 1] +
                           A[2 * N + m] * p[q - g->sy] + A[3 * N + m] * p[q + g->sy] +
                           A[4 * N + m] * p[q - g->sz] + A[5 * N + m] * p[q + g->sz];
                double ar = fabs(r);
                en = en + (norm == 2 ? ar * ar : (norm == 1 ? ar : pow(ar, norm)));
            }
    return en;
}

/* fill_coefficients, MGsolver.f90:203-251: coarse = 0.125*(sum of 8 children),
 * children summed in the order (0,0,0),(0,1,0),(0,0,1),(0,1,1),(1,0,0),
 * (1,1,0),(1,0,1),(1,1,1) in (di,dj,dk). */
static void og_fill_coefficients(const og_level* f, og_level* c) {
    static const int ord[8][3] = {{0,0,0},{0,1,0},{0,0,1},{0,1,1},{1,0,0},{1,1,0},{1,0,1},{1,1,1}};
#pragma omp parallel for collapse(2) schedule(static)
    for (int comp = 0; comp < 8; comp++)
        for (int k = 0; k < c->n[2]; k++)
            for (int j = 0; j < c->n[1]; j++)
                for (int i = 0; i < c->n[0]; i++) {
                    double s = 0.0;
                    for (int q = 0; q < 8; q++) {
                        long mf = (2 * i + ord[q][0]) + (long)f->n[0] * ((2 * j + ord[q][1]) + (long)f->n[1] * (2 * k + ord[q][2]));
                        s = q == 0 ? f->K[comp * f->N + mf] : s + f->K[comp * f->N + mf];
                    }
                    long mc = i + (long)c->n[0] * (j + (long)c->n[1] * k);
                    c->K[comp * c->N + mc] = 0.125 * s;
                }
}

/* coarse_from_fine, MGsolver.f90:185-201: Ac8 = 0; Ac8 += Af8*0.125 over
 * i1,j1,k1 = 0..1 with k1 fastest */
static void og_coarse_from_fine(const og_level* f, og_level* c) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; k++)
        for (int j = 0; j < c->n[1]; j++)
            for (int i = 0; i < c->n[0]; i++) {
                double s = 0.0;
                for (int i1 = 0; i1 < 2; i1++)
                    for (int j1 = 0; j1 < 2; j1++)
                        for (int k1 = 0; k1 < 2; k1++) {
                            long mf = (2 * i + i1) + (long)f->n[0] * ((2 * j + j1) + (long)f->n[1] * (2 * k + k1));
                            s = s + f->K[7 * f->N + mf] * 0.125;
                        }
                c->K[7 * c->N + i + (long)c->n[0] * (j + (long)c->n[1] * k)] = s;
            }
}

/* coarse_fine_interp, MGsolver.f90:128-183: piecewise-constant injection;
 * sym_MG weights the 8 children by |pf| (pf was just zeroed by the caller). */
static void og_coarse_fine_interp(const og_mg* mg, og_level* f, const og_level* c, int sym) {
    int ng = mg->g->ng;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c->n[2]; k++)
        for (int j = 0; j < c->n[1]; j++)
            for (int i = 0; i < c->n[0]; i++) {
                double pc = c->p[LIX(c, i + ng, j + ng, k + ng)];
                long q[8];
                int t = 0;
                for (int dk = 0; dk < 2; dk++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int di = 0; di < 2; di++)
                            q[t++] = LIX(f, 2 * i + di + ng, 2 * j + dj + ng, 2 * k + dk + ng);
                if (sym) {
                    /* residtot in the Fortran order of the eight terms */
                    static const int o[8] = {0, 1, 2, 3, 4, 5, 6, 7};
                    double rt = fabs(f->e[q[o[0]]]) + fabs(f->e[q[1]]) + fabs(f->e[q[2]]) + fabs(f->e[q[3]]) +
                                fabs(f->e[q[4]]) + fabs(f->e[q[5]]) + fabs(f->e[q[6]]) + fabs(f->e[q[7]]) + 1.e-15;
                    for (int s = 0; s < 8; s++) f->e[q[s]] = fabs(f->e[q[s]]) / rt * pc;
                } else {
                    for (int s = 0; s < 8; s++) f->e[q[s]] = pc;
                }
            }
}

static void og_zero(double* a, long n) {
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n; q++) a[q] = 0.0;
}

/* MG_iteration, MGsolver.f90:253-320 */
static void og_mg_iteration(og_mg* mg, double beta, int norm) {
    int LMG = mg->LMG;
    for (int L = LMG; L >= 2; L--) {
        og_level* l = &mg->lev[L];
        og_zero(l->p, l->ntot);
        for (int r = 0; r < mg->nrelax; r++) {
            og_rb_relax(mg, l, l->K, l->p, beta);
            og_apply_bc_mg(mg, l, l->p);
        }
        og_get_residual(mg, l, l->K, l->p, norm);
        og_coarse_from_fine(l, &mg->lev[L - 1]);
    }
    og_rb_relax(mg, &mg->lev[2], mg->lev[2].K, mg->lev[2].p, beta);
    og_apply_bc_mg(mg, &mg->lev[2], mg->lev[2].p);
    for (int L = 3; L <= LMG; L++) {
        og_level* l = &mg->lev[L];
        og_zero(l->e, l->ntot);
        og_coarse_fine_interp(mg, l, &mg->lev[L - 1], mg->sym);
        og_apply_bc_mg(mg, l, l->e);
        og_get_residual(mg, l, l->K, l->e, norm);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < l->ntot; q++) l->p[q] = l->p[q] + l->e[q];
        og_zero(l->e, l->ntot);
        for (int r = 0; r < mg->nrelax; r++) {
            og_rb_relax(mg, l, l->K, l->e, beta);
            og_apply_bc_mg(mg, l, l->e);
        }
#pragma omp parallel for schedule(static)
        for (long q = 0; q < l->ntot; q++) l->p[q] = l->p[q] + l->e[q];
        og_get_residual(mg, l, l->K, l->e, norm);
    }
}

/* NewSolverMG, MGsolver.f90:346-405 (via NewSolver, newsolver.f90:34-57).
 * A: 8*N (not modified); p: ghosted.  hist (optional, maxit entries) receives
 * tres2 after each V-cycle.  Returns 0, or PARIS_NOT_CONVERGED when it hits
 * maxit (it = maxit+1). */
int og_new_solver_mg_timed(const paris_grid_desc* desc, const double* A, double* p, double maxError, double beta,
                           int maxit, int norm, int* it_out, double* tres2_out, double* hist, double max_seconds);

int og_new_solver_mg(const paris_grid_desc* desc, const double* A, double* p, double maxError,
                     double beta, int maxit, int norm, int* it_out, double* tres2_out, double* hist) {
    return og_new_solver_mg_timed(desc, A, p, maxError, beta, maxit, norm, it_out, tres2_out, hist, 0.0);
}

/* NewSolverMG with a wall-clock limit (for timing runs of the host): when
 * max_seconds > 0 the loop also stops after the first V-cycle that ends past
 * max_seconds from the call, returning PARIS_NOT_CONVERGED with *it_out the
 * cycles run (not maxit+1) when the tolerance was not met. */
int og_new_solver_mg_timed(const paris_grid_desc* desc, const double* A, double* p, double maxError, double beta,
                           int maxit, int norm, int* it_out, double* tres2_out, double* hist, double max_seconds) {
    const double t_start = omp_get_wtime();
    /* init_MG, MGsolver.f90:43-46: 2^n cells per direction */
    for (int a = 0; a < 3; a++) {
        int n = a == 0 ? desc->nx : (a == 1 ? desc->ny : desc->nz);
        if (n < 2 || (n & (n - 1))) return PARIS_BAD_ARGS;
    }
    og_grid* g = og_grid_new(desc);
    og_mg* mg = og_mg_new(g);
    int LMG = mg->LMG, ng = g->ng;
    if (LMG < 2) { og_mg_free(mg); og_grid_free(g); return PARIS_BAD_ARGS; }
    og_level* lf = &mg->lev[LMG];
    long N = lf->N;
    /* get_MGmatrix_coef, MGsolver.f90:322-344 */
    memcpy(lf->K, A, 8 * N * sizeof(double));
    for (int L = LMG - 1; L >= 1; L--) og_fill_coefficients(&mg->lev[L + 1], &mg->lev[L]);
    /* initial residual with pMG(LMG) = p */
    memcpy(lf->p, p, g->ntot * sizeof(double));
    double resMax = og_get_residual(mg, lf, lf->K, lf->p, norm);
    double tres2 = resMax / (double)N;
    memset(lf->p, 0, lf->ntot * sizeof(double));
    int it;
    for (it = 1; it <= maxit; it++) {
        og_mg_iteration(mg, beta, norm);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < g->ntot; q++) p[q] = p[q] + lf->p[q];
        resMax = og_compute_residual(g, A, p, norm);
        tres2 = resMax / (double)N;
        if (norm == 2) tres2 = sqrt(tres2);
        if (hist) hist[it - 1] = tres2;
        if (tres2 < maxError) break;
        if (max_seconds > 0.0 && omp_get_wtime() - t_start > max_seconds) {
            *it_out = it;
            *tres2_out = tres2;
            og_mg_free(mg);
            og_grid_free(g);
            return PARIS_NOT_CONVERGED;
        }
    }
    (void)ng;
    *it_out = it;
    *tres2_out = tres2;
    og_mg_free(mg);
    og_grid_free(g);
    return it == maxit + 1 ? PARIS_NOT_CONVERGED : 0;
}

/* calcResidual, modules.f90:3313-3387 (ExcludeBoundCellCalcRes = F):
 * NormOrder 1 -> mean |r|, 2 -> sqrt(mean r^2), else max |r| */
double og_calc_residual(const paris_grid_desc* desc, const double* A, const double* p, int normorder) {
    og_grid* g = og_grid_new(desc);
    int ng = g->ng, nx = g->nx, ny = g->ny, nz = g->nz;
    long N = (long)nx * ny * nz;
    double res = 0.0;
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long m = i + (long)nx * (j + (long)ny * k);
                long q = OG_IX(g, i + ng, j + ng, k + ng);
                double locres = fabs(-p[q] * A[6 * N + m] + A[0 * N + m] * p[q - 1] + A[1 * N + m] * p[q + 1] +
                                     A[2 * N + m] * p[q - g->sy] + A[3 * N + m] * p[q + g->sy] +
                                     A[4 * N + m] * p[q - g->sz] + A[5 * N + m] * p[q + g->sz] + A[7 * N + m]);
                if (normorder == 1) res = res + locres;
                else if (normorder == 2) res = res + locres * locres;
                else res = res > locres ? res : locres;
            }
    double out;
    if (normorder == 1) out = res / (double)nx / (double)ny / (double)nz;
    else if (normorder == 2) out = sqrt(res / (double)nx / (double)ny / (double)nz);
    else out = res;
    og_grid_free(g);
    return out;
}

/* get_MGtest_err, MGsolver.f90:407-426: sum|p - sin sin sin| / sum|sin sin sin| */
double og_mgtest_err(const paris_grid_desc* desc, const double* p) {
    og_grid* g = og_grid_new(desc);
    const double pi = (double)3.14159265359f;
    int ng = g->ng;
    double res = 0.0, ref = 0.0;
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                double s = sin(2. * pi * g->x[i]) * sin(2. * pi * g->y[j]) * sin(2. * pi * g->z[k]);
                res = res + fabs(p[OG_IX(g, i, j, k)] - s);
                ref = ref + fabs(s);
            }
    og_grid_free(g);
    return res / ref;
}

/* project_velocity, paris.f90:882-909 (non free-surface, non STGhost):
 * u -= dt*(2*umask/dxh)*(p(i+1)-p(i))/(rho(i+1)+rho(i)) over is..ieu, etc. */
int og_project_velocity(const paris_grid_desc* desc, double* u, double* v, double* w,
                        const double* p, const double* rho, double dt) {
    og_grid* g = og_grid_new(desc);
    int ng = g->ng;
    long sy = g->sy, sz = g->sz;
    int ieu = ng + g->nx - 1, jev = ng + g->ny - 1, kew = ng + g->nz - 1;
    if (g->d.bdry_cond[0] != PARIS_BC_PERIODIC) ieu--;
    if (g->d.bdry_cond[1] != PARIS_BC_PERIODIC) jev--;
    if (g->d.bdry_cond[2] != PARIS_BC_PERIODIC) kew--;
#pragma omp parallel for schedule(static)
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i <= ieu; i++) {
                long n = OG_IX(g, i, j, k);
                u[n] = u[n] - dt * (2.0 * og_mask(g, 0, i) / g->dxh[i]) * (p[n + 1] - p[n]) / (rho[n + 1] + rho[n]);
            }
#pragma omp parallel for schedule(static)
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j <= jev; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                v[n] = v[n] - dt * (2.0 * og_mask(g, 1, j) / g->dyh[j]) * (p[n + sy] - p[n]) / (rho[n + sy] + rho[n]);
            }
#pragma omp parallel for schedule(static)
    for (int k = ng; k <= kew; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                w[n] = w[n] - dt * (2.0 * og_mask(g, 2, k) / g->dzh[k]) * (p[n + sz] - p[n]) / (rho[n + sz] + rho[n]);
            }
    og_grid_free(g);
    return 0;
}

/* ghost fill entry point for the tests (do_all_ghost) */
void og_fill_ghosts(const paris_grid_desc* desc, double* F) {
    og_grid* g = og_grid_new(desc);
    og_do_all_ghost(g, F);
    og_grid_free(g);
}
