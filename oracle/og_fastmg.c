/*
 * og_fastmg.c -- oracle (test infrastructure only): CPU restatement of the
 * B200 solver's own multigrid (the PARIS_MG_FP64 / PARIS_MG_MIXED modes),
 * which has no counterpart in the reference.  It solves the same system as
 * NewSolverMG (A from SetupPoisson, modules.f90:2735-2745; A symmetric on a
 * uniform grid, A2(i) == A1(i+1)) with:
 *   - face coefficients per level (east/north/top face of each cell), the
 *     diagonal recomputed as their sum in the order A1+..+A6;
 *   - coarse faces = mean of the four fine faces / 4 (rediscretisation);
 *   - restriction = mean of the 8 children, prolongation = injection;
 *   - red-black Gauss-Seidel V(nu1,nu2) cycles, black-red after the
 *     coarse correction (symmetric cycle), coarsest level smoothed; with a
 *     relaxation factor w != 1 each update is x + w (x_GS - x) (the
 *     reference's BETA of RedBlackRelax, newsolver.f90:229), optionally
 *     another factor on the levels below the finest; optionally
 *     nu_coarse sweeps each way on the levels coarse_from..coarse_to;
 *   - an FP64 outer loop: defect correction p += V(b - A p), or
 *     preconditioned CG with the V-cycle as preconditioner, with A applied
 *     in flux form b + sum_f a_f (x_f - x_c); CG checks the true residual
 *     when the recursive one meets the tolerance and restarts from it (at
 *     most twice) when the two have drifted apart;
 *   - inner cycle in FP32 (mixed) or FP64;
 *   - on a singular system (walls and periodic boundaries only) the initial
 *     guess with its mean taken out, the mean put back at the end.
 * The CUDA kernels of paris-git_b200/csrc/mg_fast.cu follow the same steps.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "og.h"

typedef struct {
    int n[3];
    long N;
    double *cx, *cy, *cz;   /* FP64 face coefficients */
    float *fx, *fy, *fz;    /* FP32 copies */
    double *b, *x, *r;      /* FP64 work */
    float *bf, *xf, *rf;    /* FP32 work */
    double omega;           /* relaxation factor of the red-black smoother (1: Gauss-Seidel) */
} fm_level;

typedef struct {
    int nl;
    fm_level* L;
    int per[3];
    int mixed;
    int nu1, nu2;
    int coarse_sweeps;
    int nu_coarse, coarse_from, coarse_to;   /* sweeps on the levels coarse_from..coarse_to, when nu_coarse > 0 */
} fm_mg;

/* sweeps of a smoothing pass on level L: nu, or nu_coarse on the levels coarse_from..coarse_to
 * (coarse_to <= 0: every level from coarse_from down) */
#define FM_NU(mg, L, nu)                                                                    \
    ((mg)->nu_coarse > 0 && (L) >= (mg)->coarse_from && ((mg)->coarse_to <= 0 || (L) <= (mg)->coarse_to) \
         ? (mg)->nu_coarse                                                                   \
         : (nu))

#define FIDX(l, i, j, k) ((i) + (long)(l)->n[0] * ((j) + (long)(l)->n[1] * (k)))

static inline int wrapm(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

/* neighbour value with the boundary rule: periodic wrap, wall -> the face
 * coefficient is zero so any finite value works (0). */
#define FM_NBR(T, l, per, x, i, j, k, di, dj, dk, out)                                       \
    do {                                                                                     \
        int ii = (i) + (di), jj = (j) + (dj), kk = (k) + (dk);                               \
        if ((ii < 0 || ii >= (l)->n[0]) && !per[0]) { out = (T)0; break; }                   \
        if ((jj < 0 || jj >= (l)->n[1]) && !per[1]) { out = (T)0; break; }                   \
        if ((kk < 0 || kk >= (l)->n[2]) && !per[2]) { out = (T)0; break; }                   \
        out = x[FIDX(l, wrapm(ii, (l)->n[0]), wrapm(jj, (l)->n[1]), wrapm(kk, (l)->n[2]))];  \
    } while (0)

/* face coefficient of the west/south/bottom face of a cell */
#define FM_WEST(l, per, c, i, j, k, dir)                                                     \
    ((dir) == 0 ? ((i) > 0 ? c[FIDX(l, (i) - 1, j, k)] : (per[0] ? c[FIDX(l, (l)->n[0] - 1, j, k)] : 0)) \
   : (dir) == 1 ? ((j) > 0 ? c[FIDX(l, i, (j) - 1, k)] : (per[1] ? c[FIDX(l, i, (l)->n[1] - 1, k)] : 0)) \
                : ((k) > 0 ? c[FIDX(l, i, j, (k) - 1)] : (per[2] ? c[FIDX(l, i, j, (l)->n[2] - 1)] : 0)))

#define DEF_OPS(T, SUF, CX, CY, CZ)                                                          \
static void smooth_##SUF(const fm_mg* mg, fm_level* l, const T* b, T* x, int color) {        \
    const int* per = mg->per;                                                                \
    for (int k = 0; k < l->n[2]; k++)                                                        \
        for (int j = 0; j < l->n[1]; j++)                                                    \
            for (int i = (j + k + color) & 1; i < l->n[0]; i += 2) {                         \
                long q = FIDX(l, i, j, k);                                                   \
                T a1 = FM_WEST(l, per, l->CX, i, j, k, 0), a2 = l->CX[q];                    \
                T a3 = FM_WEST(l, per, l->CY, i, j, k, 1), a4 = l->CY[q];                    \
                T a5 = FM_WEST(l, per, l->CZ, i, j, k, 2), a6 = l->CZ[q];                    \
                T pw, pe, ps, pn, pb, pt;                                                    \
                FM_NBR(T, l, per, x, i, j, k, -1, 0, 0, pw);                                 \
                FM_NBR(T, l, per, x, i, j, k, 1, 0, 0, pe);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, -1, 0, ps);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 1, 0, pn);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, -1, pb);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, 1, pt);                                  \
                T d = a1 + a2 + a3 + a4 + a5 + a6;                                           \
                T s = a1 * pw + a2 * pe + a3 * ps + a4 * pn + a5 * pb + a6 * pt + b[q];       \
                if (d > (T)0) {                                                              \
                    const T g = s / d, w = (T)l->omega;                                      \
                    x[q] = w == (T)1 ? g : x[q] + w * (g - x[q]);                            \
                }                                                                            \
            }                                                                                \
}                                                                                            \
/* r = b - A x */                                                                            \
static void resid_##SUF(const fm_mg* mg, fm_level* l, const T* b, const T* x, T* r) {        \
    const int* per = mg->per;                                                                \
    for (int k = 0; k < l->n[2]; k++)                                                        \
        for (int j = 0; j < l->n[1]; j++)                                                    \
            for (int i = 0; i < l->n[0]; i++) {                                              \
                long q = FIDX(l, i, j, k);                                                   \
                T a1 = FM_WEST(l, per, l->CX, i, j, k, 0), a2 = l->CX[q];                    \
                T a3 = FM_WEST(l, per, l->CY, i, j, k, 1), a4 = l->CY[q];                    \
                T a5 = FM_WEST(l, per, l->CZ, i, j, k, 2), a6 = l->CZ[q];                    \
                T pw, pe, ps, pn, pb, pt;                                                    \
                FM_NBR(T, l, per, x, i, j, k, -1, 0, 0, pw);                                 \
                FM_NBR(T, l, per, x, i, j, k, 1, 0, 0, pe);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, -1, 0, ps);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 1, 0, pn);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, -1, pb);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, 1, pt);                                  \
                T d = a1 + a2 + a3 + a4 + a5 + a6;                                           \
                r[q] = b[q] - d * x[q] + a1 * pw + a2 * pe + a3 * ps + a4 * pn + a5 * pb + a6 * pt; \
            }                                                                                \
}                                                                                            \
/* r = b - A x in flux form, b + sum_f a_f (x_f - x_c): the FP64 outer loop */               \
static __attribute__((unused)) void resid_flux_##SUF(const fm_mg* mg, fm_level* l, const T* b, const T* x, \
                                                      T* r) {                                \
    const int* per = mg->per;                                                                \
    for (int k = 0; k < l->n[2]; k++)                                                        \
        for (int j = 0; j < l->n[1]; j++)                                                    \
            for (int i = 0; i < l->n[0]; i++) {                                              \
                long q = FIDX(l, i, j, k);                                                   \
                T a1 = FM_WEST(l, per, l->CX, i, j, k, 0), a2 = l->CX[q];                    \
                T a3 = FM_WEST(l, per, l->CY, i, j, k, 1), a4 = l->CY[q];                    \
                T a5 = FM_WEST(l, per, l->CZ, i, j, k, 2), a6 = l->CZ[q];                    \
                T pw, pe, ps, pn, pb, pt, pc = x[q];                                         \
                FM_NBR(T, l, per, x, i, j, k, -1, 0, 0, pw);                                 \
                FM_NBR(T, l, per, x, i, j, k, 1, 0, 0, pe);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, -1, 0, ps);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 1, 0, pn);                                  \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, -1, pb);                                 \
                FM_NBR(T, l, per, x, i, j, k, 0, 0, 1, pt);                                  \
                r[q] = b[q] + (a1 * (pw - pc) + a2 * (pe - pc) + a3 * (ps - pc) + a4 * (pn - pc) + \
                               a5 * (pb - pc) + a6 * (pt - pc));                             \
            }                                                                                \
}                                                                                            \
static void restrict_##SUF(const fm_level* f, fm_level* c, const T* rf, T* bc) {             \
    for (int k = 0; k < c->n[2]; k++)                                                        \
        for (int j = 0; j < c->n[1]; j++)                                                    \
            for (int i = 0; i < c->n[0]; i++) {                                              \
                T s = 0;                                                                     \
                for (int dk = 0; dk < 2; dk++)                                               \
                    for (int dj = 0; dj < 2; dj++)                                           \
                        for (int di = 0; di < 2; di++)                                       \
                            s += rf[FIDX(f, 2 * i + di, 2 * j + dj, 2 * k + dk)];            \
                bc[FIDX(c, i, j, k)] = (T)0.125 * s;                                         \
            }                                                                                \
}                                                                                            \
static void prolong_##SUF(fm_level* f, const fm_level* c, const T* xc, T* xf) {              \
    for (int k = 0; k < f->n[2]; k++)                                                        \
        for (int j = 0; j < f->n[1]; j++)                                                    \
            for (int i = 0; i < f->n[0]; i++)                                                \
                xf[FIDX(f, i, j, k)] += xc[FIDX(c, i / 2, j / 2, k / 2)];                    \
}                                                                                            \
static void vcycle_##SUF(const fm_mg* mg, int L, T* const* B, T* const* X, T* const* R) {    \
    fm_level* l = &mg->L[L];                                                                 \
    if (L == mg->nl - 1) {                                                                   \
        for (int s = 0; s < mg->coarse_sweeps; s++) {                                        \
            smooth_##SUF(mg, l, B[L], X[L], 0);                                              \
            smooth_##SUF(mg, l, B[L], X[L], 1);                                              \
        }                                                                                    \
        for (int s = 0; s < mg->coarse_sweeps; s++) {                                        \
            smooth_##SUF(mg, l, B[L], X[L], 1);                                              \
            smooth_##SUF(mg, l, B[L], X[L], 0);                                              \
        }                                                                                    \
        return;                                                                              \
    }                                                                                        \
    for (int s = 0; s < FM_NU(mg, L, mg->nu1); s++) {                                         \
        smooth_##SUF(mg, l, B[L], X[L], 0);                                                  \
        smooth_##SUF(mg, l, B[L], X[L], 1);                                                  \
    }                                                                                        \
    resid_##SUF(mg, l, B[L], X[L], R[L]);                                                    \
    restrict_##SUF(l, &mg->L[L + 1], R[L], B[L + 1]);                                        \
    memset(X[L + 1], 0, mg->L[L + 1].N * sizeof(T));                                         \
    vcycle_##SUF(mg, L + 1, B, X, R);                                                        \
    prolong_##SUF(l, &mg->L[L + 1], X[L + 1], X[L]);                                         \
    for (int s = 0; s < FM_NU(mg, L, mg->nu2); s++) {                                         \
        smooth_##SUF(mg, l, B[L], X[L], 1);                                                  \
        smooth_##SUF(mg, l, B[L], X[L], 0);                                                  \
    }                                                                                        \
}

DEF_OPS(double, d, cx, cy, cz)
DEF_OPS(float, f, fx, fy, fz)

/* apply the V-cycle to r (FP64) -> z (FP64) */
static void precond(fm_mg* mg, const double* r, double* z) {
    fm_level* l0 = &mg->L[0];
    if (mg->mixed) {
        float* B[64]; float* X[64]; float* R[64];
        for (int L = 0; L < mg->nl; L++) { B[L] = mg->L[L].bf; X[L] = mg->L[L].xf; R[L] = mg->L[L].rf; }
        for (long q = 0; q < l0->N; q++) { B[0][q] = (float)r[q]; X[0][q] = 0.f; }
        vcycle_f(mg, 0, B, X, R);
        for (long q = 0; q < l0->N; q++) z[q] = (double)X[0][q];
    } else {
        double* B[64]; double* X[64]; double* R[64];
        for (int L = 0; L < mg->nl; L++) { B[L] = mg->L[L].b; X[L] = mg->L[L].x; R[L] = mg->L[L].r; }
        for (long q = 0; q < l0->N; q++) { B[0][q] = r[q]; X[0][q] = 0.0; }
        vcycle_d(mg, 0, B, X, R);
        for (long q = 0; q < l0->N; q++) z[q] = X[0][q];
    }
}

static double dot(const double* a, const double* b, long n) {
    double s = 0.0;
    for (long q = 0; q < n; q++) s += a[q] * b[q];
    return s;
}

/* A from SetupPoisson: fine face coefficient east = A2, north = A4, top = A6.
 * p, b: interior arrays (nx*ny*nz).  Returns cycles run; hist[it] = ||r||/||b||. */
int og_fastmg_solve(const paris_grid_desc* desc, const double* A, double* p, double rel_tol,
                    int maxit, int mixed, int pcg, int nu1, int nu2, double omega, double omega_coarse,
                    int nu_coarse, int coarse_from, int coarse_to, double* hist) {
    fm_mg mg;
    memset(&mg, 0, sizeof(mg));
    for (int a = 0; a < 3; a++) mg.per[a] = desc->bdry_cond[a] == PARIS_BC_PERIODIC;
    mg.mixed = mixed; mg.nu1 = nu1; mg.nu2 = nu2; mg.coarse_sweeps = 8;
    mg.nu_coarse = nu_coarse > 0 ? nu_coarse : 0;
    mg.coarse_from = coarse_from > 0 ? coarse_from : 1;
    mg.coarse_to = coarse_to > 0 ? coarse_to : 0;
    int n0[3] = {desc->nx, desc->ny, desc->nz};
    int nl = 1;
    while (1) {
        int m = n0[0] >> nl, mm = n0[1] >> nl, mmm = n0[2] >> nl;
        if ((n0[0] >> (nl - 1)) % 2 || (n0[1] >> (nl - 1)) % 2 || (n0[2] >> (nl - 1)) % 2) break;
        if (m < 2 || mm < 2 || mmm < 2) break;
        nl++;
    }
    mg.nl = nl;
    mg.L = calloc(nl, sizeof(fm_level));
    for (int L = 0; L < nl; L++) {
        fm_level* l = &mg.L[L];
        for (int a = 0; a < 3; a++) l->n[a] = n0[a] >> L;
        l->N = (long)l->n[0] * l->n[1] * l->n[2];
        l->omega = omega > 0.0 ? omega : 1.0;
        if (L > 0 && omega_coarse > 0.0) l->omega = omega_coarse;
        l->cx = calloc(l->N, 8); l->cy = calloc(l->N, 8); l->cz = calloc(l->N, 8);
        l->fx = calloc(l->N, 4); l->fy = calloc(l->N, 4); l->fz = calloc(l->N, 4);
        l->b = calloc(l->N, 8); l->x = calloc(l->N, 8); l->r = calloc(l->N, 8);
        l->bf = calloc(l->N, 4); l->xf = calloc(l->N, 4); l->rf = calloc(l->N, 4);
    }
    fm_level* l0 = &mg.L[0];
    long N = l0->N;
    for (long q = 0; q < N; q++) {
        l0->cx[q] = A[1 * N + q];
        l0->cy[q] = A[3 * N + q];
        l0->cz[q] = A[5 * N + q];
    }
    for (int L = 1; L < nl; L++) {
        fm_level *f = &mg.L[L - 1], *c = &mg.L[L];
        for (int k = 0; k < c->n[2]; k++)
            for (int j = 0; j < c->n[1]; j++)
                for (int i = 0; i < c->n[0]; i++) {
                    long q = FIDX(c, i, j, k);
                    int I = 2 * i + 1, J = 2 * j + 1, K = 2 * k + 1;
                    c->cx[q] = 0.0625 * (f->cx[FIDX(f, I, 2*j, 2*k)] + f->cx[FIDX(f, I, J, 2*k)] +
                                         f->cx[FIDX(f, I, 2*j, K)] + f->cx[FIDX(f, I, J, K)]);
                    c->cy[q] = 0.0625 * (f->cy[FIDX(f, 2*i, J, 2*k)] + f->cy[FIDX(f, 2*i + 1, J, 2*k)] +
                                         f->cy[FIDX(f, 2*i, J, K)] + f->cy[FIDX(f, 2*i + 1, J, K)]);
                    c->cz[q] = 0.0625 * (f->cz[FIDX(f, 2*i, 2*j, K)] + f->cz[FIDX(f, 2*i + 1, 2*j, K)] +
                                         f->cz[FIDX(f, 2*i, 2*j + 1, K)] + f->cz[FIDX(f, 2*i + 1, 2*j + 1, K)]);
                }
    }
    for (int L = 0; L < nl; L++) {
        fm_level* l = &mg.L[L];
        for (long q = 0; q < l->N; q++) {
            l->fx[q] = (float)l->cx[q]; l->fy[q] = (float)l->cy[q]; l->fz[q] = (float)l->cz[q];
        }
    }
    double* b = malloc(N * 8);
    double* r = malloc(N * 8);
    double* z = malloc(N * 8);
    double* d = malloc(N * 8);
    double* q_ = malloc(N * 8);
    for (long q = 0; q < N; q++) b[q] = A[7 * N + q];
    /* walls and periodic boundaries leave the system singular (constants
     * are its null space): solve from the initial guess with its mean taken
     * out and put the mean back at the end */
    int sing = 1;
    for (int a = 0; a < 3; a++) {
        int lo = desc->bdry_cond[a], hi = desc->bdry_cond[a + 3];
        int wall_lo = lo == PARIS_BC_WALL || lo == PARIS_BC_SHEAR, wall_hi = hi == PARIS_BC_WALL || hi == PARIS_BC_SHEAR;
        if (!mg.per[a] && !(wall_lo && wall_hi)) sing = 0;
    }
    double shift = 0.0;
    if (sing) {
        for (long q = 0; q < N; q++) shift += p[q];
        shift /= (double)N;
        for (long q = 0; q < N; q++) p[q] = p[q] - shift;
    }
    double bn = sqrt(dot(b, b, N));
    if (bn == 0.0) bn = 1.0;
    resid_flux_d(&mg, l0, b, p, r);
    double rn = sqrt(dot(r, r, N));
    int it = 0;
    if (!pcg) {
        while (it < maxit && rn / bn >= rel_tol) {
            precond(&mg, r, z);
            for (long q = 0; q < N; q++) p[q] += z[q];
            resid_flux_d(&mg, l0, b, p, r);
            rn = sqrt(dot(r, r, N));
            if (hist) hist[it] = rn / bn;
            it++;
        }
    } else {
        precond(&mg, r, z);
        memcpy(d, z, N * 8);
        double rz = dot(r, z, N);
        int restarts = 0;
        while (it < maxit && rn / bn >= rel_tol) {
            memset(q_, 0, N * 8);
            resid_flux_d(&mg, l0, q_, d, q_);   /* q_ = 0 - A d */
            for (long q = 0; q < N; q++) q_[q] = -q_[q];
            double dq = dot(d, q_, N);
            double alpha = rz / dq;
            for (long q = 0; q < N; q++) { p[q] += alpha * d[q]; r[q] -= alpha * q_[q]; }
            rn = sqrt(dot(r, r, N));
            if (hist) hist[it] = rn / bn;
            it++;
            if (rn / bn < rel_tol) {
                /* check the true residual; restart from it when rounding has
                 * let the recursive one drift away (at most twice) */
                resid_flux_d(&mg, l0, b, p, r);
                rn = sqrt(dot(r, r, N));
                if (hist) hist[it - 1] = rn / bn;
                if (rn / bn < rel_tol || restarts == 2) break;
                restarts++;
                precond(&mg, r, z);
                memcpy(d, z, N * 8);
                rz = dot(r, z, N);
                continue;
            }
            double* zold = q_;          /* reuse */
            memcpy(zold, z, N * 8);
            precond(&mg, r, z);
            double rz_new = dot(r, z, N);
            /* flexible (Polak-Ribiere) beta: r.(z - zold) / rz */
            double rzo = 0.0;
            for (long q = 0; q < N; q++) rzo += r[q] * (z[q] - zold[q]);
            double beta = rzo / rz;
            rz = rz_new;
            for (long q = 0; q < N; q++) d[q] = z[q] + beta * d[q];
        }
    }
    if (shift != 0.0)
        for (long q = 0; q < N; q++) p[q] = p[q] + shift;
    free(b); free(r); free(z); free(d); free(q_);
    for (int L = 0; L < nl; L++) {
        fm_level* l = &mg.L[L];
        free(l->cx); free(l->cy); free(l->cz); free(l->fx); free(l->fy); free(l->fz);
        free(l->b); free(l->x); free(l->r); free(l->bf); free(l->xf); free(l->rf);
    }
    free(mg.L);
    return it;
}
