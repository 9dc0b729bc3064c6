/*
 * og_adj.c -- oracle of the projection adjoint (test infrastructure only).
 *
 * The reference has no adjoint.  This file restates, in the face-coefficient
 * form B_f = 2/(rho_L + rho_R), the forward projection that SetupPoisson
 * (modules.f90:2722-2753), NewSolver and project_velocity (paris.f90:898-909)
 * compute, and its transpose:
 *   forward   A(B) p = -D u*,  u_f = u*_f - dt B_f (p_R - p_L)/dxh_f
 *   adjoint   A lambda = G^T (dt B g),
 *             g*_f = g_f + lambda_L/dx_L - lambda_R/dx_R,
 *             gB_f = -dt (p_R - p_L)/dxh_f g*_f
 * on the faces project_velocity updates (every face of a periodic direction,
 * the interior faces of a wall-bounded one).  The forward in B form lets the
 * tests take finite differences in single face coefficients.  Both solves
 * use og_fastmg_solve (FP64 PCG) on the A2/A4/A6 face coefficients.
 */
#include <math.h>
#include <string.h>

#include "og.h"

int og_fastmg_solve(const paris_grid_desc* desc, const double* A, double* p, double rel_tol, int maxit,
                    int mixed, int pcg, int nu1, int nu2, double omega, double omega_coarse, int nu_coarse,
                    int coarse_from, int coarse_to, double* hist);

typedef struct {
    og_grid* g;
    int n[3], per[3];
    long st[3];
    const double *dx[3], *dxh[3];
} adj_geo;

static void geo_init(adj_geo* a, og_grid* g) {
    a->g = g;
    for (int d = 0; d < 3; d++) {
        a->n[d] = g->N[d];
        a->per[d] = og_is_periodic(g, d);
    }
    a->st[0] = 1; a->st[1] = g->sy; a->st[2] = g->sz;
    a->dx[0] = g->dx; a->dx[1] = g->dy; a->dx[2] = g->dz;
    a->dxh[0] = g->dxh; a->dxh[1] = g->dyh; a->dxh[2] = g->dzh;
}

/* face f (interior-relative) of direction d is updated by the projection */
static int owned(const adj_geo* a, int d, int f) { return f < a->n[d] - 1 || a->per[d]; }

/* B_f = 2/(rho_f + rho_{f+1}) on the updated faces, reading the ghost layer
 * as project_velocity does; 0 elsewhere */
void og_face_B(const paris_grid_desc* desc, const double* rho, double* Bx, double* By, double* Bz) {
    og_grid* g = og_grid_new(desc);
    adj_geo a;
    geo_init(&a, g);
    double* B[3] = {Bx, By, Bz};
    int ng = g->ng;
    for (int d = 0; d < 3; d++) memset(B[d], 0, g->ntot * sizeof(double));
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                for (int d = 0; d < 3; d++)
                    if (owned(&a, d, ix[d])) B[d][n] = 2.0 / (rho[n + a.st[d]] + rho[n]);
            }
    og_grid_free(g);
}

/* A2/A4/A6 (east/north/top coefficient of every cell) of SetupPoisson in the
 * B form: dt B_f / (dx_c dxh_f), zero on wall faces */
static void face_matrix(const adj_geo* a, double dt, double* const B[3], double* A) {
    og_grid* g = a->g;
    int ng = g->ng;
    long N = (long)g->nx * g->ny * g->nz;
    memset(A, 0, 8 * N * sizeof(double));
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                long t = i + (long)g->nx * (j + (long)g->ny * k);
                for (int d = 0; d < 3; d++)
                    if (owned(a, d, ix[d]))
                        A[(2 * d + 1) * N + t] = dt * B[d][n] / (a->dx[d][ix[d] + ng] * a->dxh[d][ix[d] + ng]);
            }
}

static void interior_to_ghosted(og_grid* g, const double* x, double* p) {
    int ng = g->ng;
    memset(p, 0, g->ntot * sizeof(double));
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++)
                p[OG_IX(g, i + ng, j + ng, k + ng)] = x[i + (long)g->nx * (j + (long)g->ny * k)];
    og_do_all_ghost(g, p);
}

/* Forward projection in the B form.  us: u*, v*, w* (ghosted; the updated
 * faces are the unknowns, the wall faces are read as constants); uo: the
 * projected velocity on the updated faces (other entries copied from us);
 * p: the pressure with periodic ghosts.  Returns the solver's cycle count. */
int og_projection_forward_B(const paris_grid_desc* desc, double dt, const double* Bx, const double* By,
                            const double* Bz, const double* us, const double* vs, const double* ws, double* uo,
                            double* vo, double* wo, double* p, double rel_tol, int maxit) {
    og_grid* g = og_grid_new(desc);
    adj_geo a;
    geo_init(&a, g);
    int ng = g->ng;
    long N = (long)g->nx * g->ny * g->nz;
    double* B[3] = {(double*)Bx, (double*)By, (double*)Bz};
    const double* U[3] = {us, vs, ws};
    double* O[3] = {uo, vo, wo};
    double* A = malloc(8 * N * sizeof(double));
    double* x = calloc(N, sizeof(double));
    face_matrix(&a, dt, B, A);
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                long t = i + (long)g->nx * (j + (long)g->ny * k);
                double div = 0.0;
                for (int d = 0; d < 3; d++) {
                    /* west face: the periodic image of face n-1 at the seam */
                    long nw = n - a.st[d];
                    if (ix[d] == 0 && a.per[d]) nw = n + (long)(a.n[d] - 1) * a.st[d];
                    div += (U[d][n] - U[d][nw]) / a.dx[d][ix[d] + ng];
                }
                A[7 * N + t] = -div;
            }
    int it = og_fastmg_solve(desc, A, x, rel_tol, maxit, 0, 1, 2, 2, 1.0, 0.0, 0, 1, 0, NULL);
    interior_to_ghosted(g, x, p);
    for (int d = 0; d < 3; d++) memcpy(O[d], U[d], g->ntot * sizeof(double));
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                for (int d = 0; d < 3; d++)
                    if (owned(&a, d, ix[d]))
                        O[d][n] = U[d][n] - dt * B[d][n] * (p[n + a.st[d]] - p[n]) / a.dxh[d][ix[d] + ng];
            }
    free(A);
    free(x);
    og_grid_free(g);
    return it;
}

/* The adjoint.  B: face coefficients (og_face_B); p: the forward pressure
 * with ghosts; gu..: dL/du; outputs dL/du* and dL/dB on the updated faces,
 * zero elsewhere.  Returns the cycle count of the transpose solve. */
int og_projection_adjoint(const paris_grid_desc* desc, double dt, const double* Bx, const double* By,
                          const double* Bz, const double* p, const double* gu, const double* gv, const double* gw,
                          double* su, double* sv, double* sw, double* bx, double* by, double* bz, double rel_tol,
                          int maxit) {
    og_grid* g = og_grid_new(desc);
    adj_geo a;
    geo_init(&a, g);
    int ng = g->ng;
    long N = (long)g->nx * g->ny * g->nz;
    double* B[3] = {(double*)Bx, (double*)By, (double*)Bz};
    const double* G[3] = {gu, gv, gw};
    double* S[3] = {su, sv, sw};
    double* BO[3] = {bx, by, bz};
    double* A = malloc(8 * N * sizeof(double));
    double* x = calloc(N, sizeof(double));
    double* lam = malloc(g->ntot * sizeof(double));
    face_matrix(&a, dt, B, A);
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                long t = i + (long)g->nx * (j + (long)g->ny * k);
                double s = 0.0;
                for (int d = 0; d < 3; d++) {
                    int c = ix[d], nd = a.n[d];
                    if (owned(&a, d, c)) s -= dt * B[d][n] * G[d][n] / a.dxh[d][c + ng];
                    if (c > 0 || a.per[d]) {
                        int fw = c > 0 ? c - 1 : nd - 1;
                        long nf = n + (long)(fw - c) * a.st[d];
                        s += dt * B[d][nf] * G[d][nf] / a.dxh[d][fw + ng];
                    }
                }
                A[7 * N + t] = s;
            }
    int it = og_fastmg_solve(desc, A, x, rel_tol, maxit, 0, 1, 2, 2, 1.0, 0.0, 0, 1, 0, NULL);
    interior_to_ghosted(g, x, lam);
    for (int d = 0; d < 3; d++) {
        memset(S[d], 0, g->ntot * sizeof(double));
        memset(BO[d], 0, g->ntot * sizeof(double));
    }
    for (int k = 0; k < g->nz; k++)
        for (int j = 0; j < g->ny; j++)
            for (int i = 0; i < g->nx; i++) {
                int ix[3] = {i, j, k};
                long n = OG_IX(g, i + ng, j + ng, k + ng);
                for (int d = 0; d < 3; d++) {
                    int c = ix[d], nd = a.n[d];
                    if (!owned(&a, d, c)) continue;
                    int cr = c < nd - 1 ? c + 1 : 0;
                    long nr = n + (long)(cr - c) * a.st[d];
                    double gs = G[d][n] + lam[n] / a.dx[d][c + ng] - lam[nr] / a.dx[d][cr + ng];
                    S[d][n] = gs;
                    BO[d][n] = -dt * (p[n + a.st[d]] - p[n]) / a.dxh[d][c + ng] * gs;
                }
            }
    free(A);
    free(x);
    free(lam);
    og_grid_free(g);
    return it;
}
