/*
 * og_grid.c -- oracle (test infrastructure only): grid coordinates and the
 * single-rank ghost exchange of the reference.
 */
#include <string.h>
#include "og.h"

/* Uniform grid of the reference, paris.f90:3057-3100 with xform=0:
 *   xh(i) = xLength*(xform*s*(0.5-s)*(1-s)+s), s=(i-Ng)/Nx
 *   x(i)  = 0.5*(xh(i)+xh(i-1)), x(1)=2*xh(1)-x(2)
 *   dxh(i)= x(i+1)-x(i), dxh(Nxt)=dxh(Nxt-1)
 *   dx(i) = xh(i)-xh(i-1), dx(1)=dx(2)                                       */
static void og_axis(int n, int ng, double L, double** px, double** pxh, double** pdx,
                    double** pdxh) {
    int nt = n + 2 * ng;
    double* x = calloc(nt, sizeof(double));
    double* xh = calloc(nt, sizeof(double));
    double* dx = calloc(nt, sizeof(double));
    double* dxh = calloc(nt, sizeof(double));
    const double form = 0.0;
    for (int f = 1; f <= nt; f++) {
        double s = (double)(f - ng) / (double)n;
        xh[f - 1] = L * (form * s * (0.5 - s) * (1.0 - s) + s);
    }
    for (int f = 2; f <= nt; f++) x[f - 1] = 0.5 * (xh[f - 1] + xh[f - 2]);
    x[0] = 2.0 * xh[0] - x[1];
    for (int f = 1; f <= nt - 1; f++) dxh[f - 1] = x[f] - x[f - 1];
    dxh[nt - 1] = dxh[nt - 2];
    for (int f = 2; f <= nt; f++) dx[f - 1] = xh[f - 1] - xh[f - 2];
    dx[0] = dx[1];
    *px = x; *pxh = xh; *pdx = dx; *pdxh = dxh;
}

og_grid* og_grid_new(const paris_grid_desc* d) {
    og_grid* g = calloc(1, sizeof(og_grid));
    g->d = *d;
    g->nx = d->nx; g->ny = d->ny; g->nz = d->nz; g->ng = d->ng;
    g->N[0] = d->nx; g->N[1] = d->ny; g->N[2] = d->nz;
    for (int a = 0; a < 3; a++) g->Nt[a] = g->N[a] + 2 * g->ng;
    g->sy = g->Nt[0];
    g->sz = (long)g->Nt[0] * g->Nt[1];
    g->ntot = g->sz * g->Nt[2];
    og_axis(d->nx, d->ng, d->xlength, &g->x, &g->xh, &g->dx, &g->dxh);
    og_axis(d->ny, d->ng, d->ylength, &g->y, &g->yh, &g->dy, &g->dyh);
    og_axis(d->nz, d->ng, d->zlength, &g->z, &g->zh, &g->dz, &g->dzh);
    return g;
}

void og_grid_free(og_grid* g) {
    if (!g) return;
    free(g->x); free(g->xh); free(g->dx); free(g->dxh);
    free(g->y); free(g->yh); free(g->dy); free(g->dyh);
    free(g->z); free(g->zh); free(g->dz); free(g->dzh);
    free(g);
}

int og_is_periodic(const og_grid* g, int dir) {
    return g->d.bdry_cond[dir] == PARIS_BC_PERIODIC;
}

/* ghost_x/y/z (modules.f90:1821-1970) on a single rank: the Cartesian
 * neighbour is the rank itself for a periodic direction, so the receive of
 * F(is-ngh:is-1) gets F(ie-ngh+1:ie) and F(ie+1:ie+ngh) gets F(is:is+ngh-1),
 * over the full extent of the other two directions; for a wall the neighbour
 * is MPI_PROC_NULL and nothing is written. */
#define OG_GHOST_BODY(T)                                                              \
    if (!og_is_periodic(g, dir)) return;                                              \
    int n = g->N[dir], ng = g->ng;                                                    \
    int lo = ng, hi = ng + n - 1;                                                     \
    int o1 = (dir + 1) % 3, o2 = (dir + 2) % 3;                                       \
    long st[3] = {1, g->sy, g->sz};                                                   \
    for (int b = 0; b < g->Nt[o2]; b++)                                               \
        for (int a = 0; a < g->Nt[o1]; a++) {                                         \
            T* base = F + a * st[o1] + b * st[o2];                                    \
            for (int l = 1; l <= ngh; l++) {                                          \
                base[(lo - l) * st[dir]] = base[(hi - l + 1) * st[dir]];              \
                base[(hi + l) * st[dir]] = base[(lo + l - 1) * st[dir]];              \
            }                                                                         \
        }

void og_ghost_dir(const og_grid* g, double* F, int dir, int ngh) { OG_GHOST_BODY(double) }
void og_ighost_dir(const og_grid* g, int32_t* F, int dir, int ngh) { OG_GHOST_BODY(int32_t) }

void og_do_all_ghost(const og_grid* g, double* F) {
    for (int d = 0; d < 3; d++) og_ghost_dir(g, F, d, 2);
}
void og_do_all_ighost(const og_grid* g, int32_t* F) {
    for (int d = 0; d < 3; d++) og_ighost_dir(g, F, d, 2);
}
