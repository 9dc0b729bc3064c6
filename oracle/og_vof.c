/*
 * og_vof.c -- oracle (test infrastructure only): split VOF advection,
 * flags/clipping, VOF boundary conditions, linfunc and the level-set
 * initialisation, restated from vofnonmodule.f90 and vofmodules.f90.
 */
#include <math.h>
#include <string.h>
#include "og.h"

/* inject(j,k) of SetVOFBC, vofmodules.f90:1797-1811 (j,k ghosted C indices) */
static int og_inject(const og_grid* g, int j, int k) {
    const paris_grid_desc* d = &g->d;
    double yy = g->y[j] - d->jetcenter_yc, zz = g->z[k] - d->jetcenter_zc;
    if (d->inject_type == 2 || d->inject_type == 4) {
        if (yy * yy + zz * zz < d->radius_liq_inject * d->radius_liq_inject) return 1;
    } else if (d->inject_type == 3) {
        if (yy <= d->radius_liq_inject) return 1;
    } else if (d->inject_type == 5) {
        if (yy > d->radius_gas_inject && yy < d->radius_liq_inject) return 1;
    }
    return 0;
}

/* SetVOFBC, vofmodules.f90:1694-1825: orientations x- y- z- x+ y+ z+ in
 * turn, each over the whole ghosted extent of the other two directions.
 * 'dry'/'wet' set both ghost layers, 'outflow' copies the boundary cell into
 * both; 'jet' (x- only) sets the first layer to inject(j,k) and '90deg' the
 * first layer to the adjacent cell, leaving the second layer as it was. */
void og_setvofbc(const og_grid* g, double* cv, int32_t* fl) {
    for (int orient = 0; orient < 6; orient++) {
        int cond = g->d.vofbdry_cond[orient];
        int d = orient % 3;
        int sign = orient < 3 ? -1 : 1;
        if (cond == PARIS_VOFBC_PERIODIC) continue;
        int t2 = (d + 1) % 3, t3 = (d + 2) % 3;
        if (t2 > t3) { int t = t2; t2 = t3; t3 = t; }
        int lim = sign < 0 ? g->ng : g->ng + g->N[d] - 1;   /* coordlimit */
        long st[3] = {1, g->sy, g->sz};
        for (int l = 0; l < g->Nt[t2]; l++)
            for (int m = 0; m < g->Nt[t3]; m++) {
                long base = l * st[t2] + m * st[t3];
                long g1 = base + (long)(lim + sign) * st[d];
                long g2 = base + (long)(lim + 2 * sign) * st[d];
                long in = base + (long)lim * st[d];
                if (cond == PARIS_VOFBC_DRY || cond == PARIS_VOFBC_WET) {
                    int flag = cond == PARIS_VOFBC_WET ? 1 : 0;
                    cv[g1] = (double)flag; fl[g1] = flag;
                    cv[g2] = (double)flag; fl[g2] = flag;
                } else if (cond == PARIS_VOFBC_JET) {
                    /* c(2) = l, c(3) = m: t2 = y, t3 = z for the x- face */
                    int inj = og_inject(g, l, m);
                    cv[g1] = (double)inj; fl[g1] = inj;
                } else if (cond == PARIS_VOFBC_OUTFLOW) {
                    double cvh = cv[in]; int32_t flh = fl[in];
                    cv[g1] = cvh; fl[g1] = flh;
                    cv[g2] = cvh; fl[g2] = flh;
                } else if (cond == PARIS_VOFBC_90DEG) {
                    cv[g1] = cv[in]; fl[g1] = fl[in];
                }
            }
    }
}

/* get_flags_and_clip, vofmodules.f90:549-571 (all cells, ghosts included) */
void og_flags_and_clip(const og_grid* g, double* c, int32_t* f) {
    double epsc = g->d.epsc;
    for (long n = 0; n < g->ntot; n++) {
        if (c[n] <= epsc) {
            f[n] = 0; c[n] = 0.0;
        } else if (c[n] >= 1.0 - epsc) {
            f[n] = 1; c[n] = 1.0;
        } else {
            f[n] = 2;
        }
    }
}

/* get_vof_phase, vofmodules.f90:573-592 */
void og_vof_phase(const og_grid* g, const double* c, int32_t* phase) {
    double epsc = g->d.epsc;
    for (long n = 0; n < g->ntot; n++) phase[n] = c[n] < (0.5 - epsc) ? 0 : 1;
}

void og_stencil(const og_grid* g, const double* c, long n, double st[27]) {
    for (int i1 = -1; i1 <= 1; i1++)
        for (int j1 = -1; j1 <= 1; j1++)
            for (int k1 = -1; k1 <= 1; k1++)
                st[OG_C3(i1 + 1, j1 + 1, k1 + 1)] = c[n + i1 + j1 * g->sy + k1 * g->sz];
}

/* fit_plane_new, vofnonmodule.f90:633-655; returns 1 on error (zero normal) */
int og_fit_plane_new(double vof, int d, double a1, double a2, const double st[27],
                            double m[3], double* alpha) {
    og_mycs(st, m);
    if (m[0] == 0.0 && m[1] == 0.0 && m[2] == 0.0) return 1;
    *alpha = og_al3d(m, vof);
    m[d] = m[d] / (1.0 - a1 + a2);
    *alpha = *alpha + m[d] * a1;
    return 0;
}

/* swpz (CIAM, Lagrangian explicit), vofnonmodule.f90:126-237.
 * us: face velocity in direction d; v1,v2,v3 work arrays. */
static void og_swpz(const og_grid* g, const double* us, double* c, int32_t* f, int d,
                    double dt, double* v1, double* v2, double* v3) {
    long st[3] = {1, g->sy, g->sz};
    long o = st[d];
    double dxyz = g->dxh[g->ng];   /* dxyz = dxh(is) for every direction (cubic cells) */
    int ng = g->ng;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng - 1; k <= ng + g->nz; k++)
        for (int j = ng - 1; j <= ng + g->ny; j++)
            for (int i = ng - 1; i <= ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                double a2 = us[n] * dt / dxyz;
                double a1 = us[n - o] * dt / dxyz;
                v1[n] = 0.0; v2[n] = 0.0; v3[n] = 0.0;
                if (c[n] == 1.0) {
                    v1[n] = og_dmax1(-a1, 0.0);
                    v2[n] = 1.0 - og_dmax1(a1, 0.0) + og_dmin1(a2, 0.0);
                    v3[n] = og_dmax1(a2, 0.0);
                } else if (c[n] > 0.0) {
                    double s[27], nr[3], alpha, x0[3], dx[3];
                    og_stencil(g, c, n, s);
                    if (og_fit_plane_new(c[n], d, a1, a2, s, nr, &alpha)) continue;
                    double mm1 = og_dmax1(a1, 0.0);
                    double mm2 = 1.0 - mm1 + og_dmin1(0.0, a2);
                    x0[0] = x0[1] = x0[2] = 0.0;
                    dx[0] = dx[1] = dx[2] = 1.0;
                    if (a1 < 0.0) {
                        x0[d] = a1;
                        dx[d] = -a1;
                        v1[n] = og_fl3d(nr, alpha, x0, dx);
                    }
                    if (a2 > 0.0) {
                        x0[d] = 1.0;
                        dx[d] = a2;
                        v3[n] = og_fl3d(nr, alpha, x0, dx);
                    }
                    x0[d] = mm1;
                    dx[d] = mm2;
                    v2[n] = og_fl3d(nr, alpha, x0, dx);
                }
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                double cn = v3[n - o] + v2[n] + v1[n + o];
                c[n] = og_dmax1(0.0, og_dmin1(1.0, cn));
            }
    og_setvofbc(g, c, f);
}

/* swpr (Weymouth-Yue, Eulerian implicit + central term), vofnonmodule.f90:664-754.
 * cg: c_mask of cvof frozen before the three sweeps. */
static void og_swpr(const og_grid* g, const double* us, double* c, int32_t* f, int d,
                    double dt, double* v1, const double* cg, double* v3) {
    long st[3] = {1, g->sy, g->sz};
    long o = st[d];
    double dxyz = g->dxh[g->ng];
    int ng = g->ng;
    double epsc = g->d.epsc;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng - 1; k <= ng + g->nz; k++)
        for (int j = ng - 1; j <= ng + g->ny; j++)
            for (int i = ng - 1; i <= ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                double a2 = us[n] * dt / dxyz;
                double a1 = us[n - o] * dt / dxyz;
                v1[n] = 0.0; v3[n] = 0.0;
                if (c[n] == 1.0) {
                    v1[n] = og_dmax1(-a1, 0.0);
                    v3[n] = og_dmax1(a2, 0.0);
                } else if (c[n] > 0.0) {
                    double s[27], m[3], x0[3], dx[3];
                    og_stencil(g, c, n, s);
                    og_mycs(s, m);
                    double alpha = og_al3d(m, c[n]);
                    x0[0] = x0[1] = x0[2] = 0.0;
                    dx[0] = dx[1] = dx[2] = 1.0;
                    if (a1 < 0.0) {
                        dx[d] = -a1;
                        v1[n] = og_fl3d(m, alpha, x0, dx);
                    }
                    if (a2 > 0.0) {
                        x0[d] = 1.0 - a2;
                        dx[d] = a2;
                        v3[n] = og_fl3d(m, alpha, x0, dx);
                    }
                }
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                double a2 = us[n] * dt / dxyz;
                double a1 = us[n - o] * dt / dxyz;
                double cn = c[n] - (v3[n] - v1[n + o]) + (v3[n - o] - v1[n]) + cg[n] * (a2 - a1);
                if (cn < epsc) cn = 0.0;
                else if (cn > 1.0 - epsc) cn = 1.0;
                c[n] = cn;
            }
    og_setvofbc(g, c, f);
}

/* swp, vofnonmodule.f90:27-48 */
void og_swp(const og_grid* g, const double* us, double* c, int32_t* f, int d, double dt,
                   double* w1, double* w2, double* w3, int32_t* phase) {
    if (g->d.vof_advect == PARIS_ADVECT_WY)
        og_swpr(g, us, c, f, d, dt, w1, w2, w3);
    else
        og_swpz(g, us, c, f, d, dt, w1, w2, w3);
    og_do_all_ghost(g, c);
    og_flags_and_clip(g, c, f);
    og_do_all_ighost(g, f);
    if (phase) og_vof_phase(g, c, phase);
}

/* vofsweeps(tswap), vofmodules.f90:1340-1361. Arrays are ghosted. */
int og_vofsweeps(const paris_grid_desc* desc, int tswap, double dt, double* cvof, int32_t* flag,
                 int32_t* phase, const double* u, const double* v, const double* w) {
    og_grid* g = og_grid_new(desc);
    double* w1 = calloc(g->ntot, sizeof(double));
    double* w2 = calloc(g->ntot, sizeof(double));
    double* w3 = calloc(g->ntot, sizeof(double));
    if (g->d.vof_advect == PARIS_ADVECT_WY)   /* c_mask(cvof, work(:,:,:,2)), vofmodules.f90:1295 */
        for (long n = 0; n < g->ntot; n++) w2[n] = cvof[n] > 0.5 ? 1.0 : 0.0;
    const double* vel[3] = {u, v, w};
    int order[3];
    if (tswap % 3 == 0) { order[0] = 2; order[1] = 0; order[2] = 1; }
    else if (tswap % 3 == 1) { order[0] = 1; order[1] = 2; order[2] = 0; }
    else { order[0] = 0; order[1] = 1; order[2] = 2; }
    for (int s = 0; s < 3; s++)
        og_swp(g, vel[order[s]], cvof, flag, order[s], dt, w1, w2, w3, phase);
    free(w1); free(w2); free(w3);
    og_grid_free(g);
    return 0;
}

/* c_mask, get_flags_and_clip entry points for the tests */
int og_flags_clip(const paris_grid_desc* desc, double* c, int32_t* f) {
    og_grid* g = og_grid_new(desc);
    og_flags_and_clip(g, c, f);
    og_grid_free(g);
    return 0;
}

/* linfunc(field,a1,a2,MeanFlag), vofmodules.f90:171-218 (+ initialize_linfunc :133) */
int og_linfunc(const paris_grid_desc* desc, double* field, const double* cvof, double a1,
               double a2, int meanflag) {
    og_grid* g = og_grid_new(desc);
    const double b1 = 8.0 / 64, b2 = 4.0 / 64, b3 = 2.0 / 64, b4 = 1.0 / 64;
    double inva1 = 0.0, inva2 = 0.0;
    if (meanflag == PARIS_MEAN_HARM) {
        inva1 = 1.0 / (a1 + 1e-50);
        inva2 = 1.0 / (a2 + 1e-50);
    }
    if (g->d.nfilter == 0) {
        for (long n = 0; n < g->ntot; n++) {
            if (meanflag == PARIS_MEAN_ARITH) field[n] = cvof[n] * (a2 - a1) + a1;
            else field[n] = 1.0 / (cvof[n] * (inva2 - inva1) + inva1);
        }
    } else {
        long sy = g->sy, sz = g->sz;
        for (int k = 0; k < g->Nt[2]; k++)
            for (int j = 0; j < g->Nt[1]; j++)
                for (int i = 0; i < g->Nt[0]; i++) {
                    long n = OG_IX(g, i, j, k);
                    const double* c = cvof;
                    double cf;
                    if (k > 0 && k < g->Nt[2] - 1 && j > 0 && j < g->Nt[1] - 1 && i > 0 && i < g->Nt[0] - 1) {
                        cf = b1 * c[n] +
                             b2 * (c[n - 1] + c[n - sy] + c[n - sz] + c[n + 1] + c[n + sy] + c[n + sz]) +
                             b3 * (c[n + 1 + sy] + c[n + 1 - sy] + c[n - 1 + sy] + c[n - 1 - sy] +
                                   c[n + 1 + sz] + c[n + 1 - sz] + c[n - 1 + sz] + c[n - 1 - sz] +
                                   c[n + sy + sz] + c[n + sy - sz] + c[n - sy + sz] + c[n - sy - sz]) +
                             b4 * (c[n + 1 + sy + sz] + c[n + 1 + sy - sz] + c[n + 1 - sy + sz] + c[n + 1 - sy - sz] +
                                   c[n - 1 + sy + sz] + c[n - 1 + sy - sz] + c[n - 1 - sy + sz] + c[n - 1 - sy - sz]);
                    } else {
                        cf = c[n];
                    }
                    if (meanflag == PARIS_MEAN_ARITH) field[n] = cf * (a2 - a1) + a1;
                    else field[n] = 1.0 / (cf * (inva2 - inva1) + inva1);
                }
    }
    og_do_all_ghost(g, field);
    og_grid_free(g);
    return 0;
}

/* ls2vof_in_cell, vofnonmodule.f90:1142-1190 */
static double og_ls2vof_in_cell(const double st[27], int* nflag) {
    double m[3], zero[3] = {0, 0, 0}, one[3] = {1, 1, 1};
    og_fd32(st, m);
    m[0] = fabs(m[0]); m[1] = fabs(m[1]); m[2] = fabs(m[2]);
    double norml1 = m[0] + m[1] + m[2];
    m[0] = m[0] / norml1; m[1] = m[1] / norml1; m[2] = m[2] / norml1;
    double alpha = 32.0 * st[OG_C3(1, 1, 1)] / norml1;
    alpha = alpha + 0.5;
    if (alpha >= 1.0) { *nflag = 1; return 1.0; }
    if (alpha <= 0.0) { *nflag = 0; return 0.0; }
    *nflag = 2;
    return og_fl3d(m, alpha, zero, one);
}

typedef struct {
    int nb;
    const double *xc, *yc, *zc, *rad;
    double cdir[3];   /* 1/(1 + excentricity), 0 along a cylinder's axis */
    int prune;        /* spheres (cdir = 1): candidate bubbles per cell */
    int wave;         /* wave2ls instead of shapes2ls */
    double hdir[3], vdir[3], len[3], amp, shift, nsign;
    int ncand;
    int cand[4096];
} og_spheres;

/* shapes2ls, vofmodules.f90:973-993: max over bubbles of rad^2 -
 * sum_a cdir(a) (x_a - xc_a)^2, cdir = 1/(1 + excentricity) with the
 * cylinder axis (ipar < 0) zeroed.  For spheres the max runs over the
 * candidate bubbles of the current cell only; og_candidates() keeps every
 * bubble that can reach the max anywhere in the cell's stencil region, so the
 * value is the same as the max over all bubbles. */
/* wave2ls, vofmodules.f90:997-1034: a cosine interface normal to vdir,
 * varying along hdir, with amplitude 0.5*A_h*dx(nx/2+2) */
static double og_wave2ls(const og_spheres* s, double xx, double yy, double zz) {
    const double PI = 3.14159265359;   /* module_grid PI */
    double w = s->vdir[2] * (-zz + s->len[2] / 2.0) + s->vdir[1] * (-yy + s->len[1] / 2.0) +
               s->vdir[0] * (-xx + s->len[0] / 2.0) +
               s->amp * cos(2.0 * PI * (s->hdir[0] * xx / s->len[0] + s->hdir[1] * yy / s->len[1] +
                                        s->hdir[2] * zz / s->len[2]));
    return w * s->nsign + s->shift;
}

static double og_shapes2ls(const og_spheres* s, double xx, double yy, double zz) {
    if (s->wave) return og_wave2ls(s, xx, yy, zz);
    double r = -2.0e6;
    for (int q = 0; q < s->ncand; q++) {
        int ib = s->cand[q];
        double v = s->rad[ib] * s->rad[ib] -
                   (s->cdir[0] * ((xx - s->xc[ib]) * (xx - s->xc[ib])) +
                    s->cdir[1] * ((yy - s->yc[ib]) * (yy - s->yc[ib])) +
                    s->cdir[2] * ((zz - s->zc[ib]) * (zz - s->zc[ib])));
        r = r > v ? r : v;
    }
    return r;
}

/* bubbles whose upper bound of rad^2 - d^2 over the sphere (c, R) reaches the
 * best lower bound; the others can never be the max there. */
static void og_candidates(og_spheres* s, double cx, double cy, double cz, double R) {
    double ub[4096], lbmax = -1e300;
    int nb = s->nb < 4096 ? s->nb : 4096;
    for (int ib = 0; ib < nb; ib++) {
        double dx = cx - s->xc[ib], dy = cy - s->yc[ib], dz = cz - s->zc[ib];
        double D = sqrt(dx * dx + dy * dy + dz * dz);
        double r2 = s->rad[ib] * s->rad[ib];
        double dn = D - R > 0.0 ? D - R : 0.0;
        ub[ib] = r2 - dn * dn;
        double lb = r2 - (D + R) * (D + R);
        if (lb > lbmax) lbmax = lb;
    }
    s->ncand = 0;
    for (int ib = 0; ib < nb; ib++)
        if (ub[ib] >= lbmax - 1e-9 * (fabs(lbmax) + 1.0)) s->cand[s->ncand++] = ib;
}

/* notisolated, vofmodules.f90:1126-1150 (3-D case) */
static int og_notisolated(const int32_t is3[27]) {
    int nfrac = 0, nfull = 0, ncells = 0;
    for (int q = 0; q < 27; q++) {
        nfrac += is3[q] / 2;
        nfull += is3[q] % 2;
        ncells++;
    }
    return !(nfrac == 0 && (nfull == 0 || nfull == ncells));
}

/* ls2vof_refined, vofmodules.f90:1195-1293, for spheres (d = 0) */
static void og_ls2vof_refined(const og_grid* g, og_spheres* s, int n1, double* cvof,
                              int32_t* flag, const int32_t* fin) {
    int ng = g->ng;
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                int refinethis = 0;
                if (n1 > 1) {
                    int32_t is3[27];
                    for (int i0 = -1; i0 <= 1; i0++)
                        for (int j0 = -1; j0 <= 1; j0++)
                            for (int k0 = -1; k0 <= 1; k0++)
                                is3[OG_C3(i0 + 1, j0 + 1, k0 + 1)] = fin[n + i0 + j0 * g->sy + k0 * g->sz];
                    refinethis = og_notisolated(is3);
                }
                if (n1 == 1 || refinethis) {
                    double dx1 = g->dx[i] / n1, dy1 = g->dy[j] / n1, dz1 = g->dz[k] / n1;
                    if (s->prune) {   /* stencil points lie within half a cell plus one sub-cell of the centre */
                        double hx = 0.5 * g->dx[i] + dx1, hy = 0.5 * g->dy[j] + dy1, hz = 0.5 * g->dz[k] + dz1;
                        og_candidates(s, g->x[i], g->y[j], g->z[k], 1.000001 * sqrt(hx * hx + hy * hy + hz * hz));
                    }
                    int nfrac = 0, nfull = 0;
                    double b = 0.0;
                    for (int l = 0; l < n1; l++)
                        for (int m = 0; m < n1; m++)
                            for (int q = 0; q < n1; q++) {
                                double x0 = g->x[i] - 0.5 * g->dx[i] + 0.5 * dx1 + dx1 * l;
                                double y0 = g->y[j] - 0.5 * g->dy[j] + 0.5 * dy1 + dy1 * m;
                                double z0 = g->z[k] - 0.5 * g->dz[k] + 0.5 * dz1 + dz1 * q;
                                double st[27];
                                for (int i0 = -1; i0 <= 1; i0++)
                                    for (int j0 = -1; j0 <= 1; j0++)
                                        for (int k0 = -1; k0 <= 1; k0++) {
                                            double x1 = x0 + i0 * dx1, y1 = y0 + j0 * dy1, z1 = z0 + k0 * dz1;
                                            st[OG_C3(i0 + 1, j0 + 1, k0 + 1)] = og_shapes2ls(s, x1, y1, z1);
                                        }
                                int nflag;
                                double a = og_ls2vof_in_cell(st, &nflag);
                                if (nflag == 2) nfrac++;
                                else if (nflag == 1) nfull++;
                                b = b + a;
                            }
                    cvof[n] = b / (double)(n1 * n1 * n1);
                    if (nfrac > 0) {
                        flag[n] = 2;
                    } else if (nfull == n1 * n1 * n1) {
                        flag[n] = 1;
                        cvof[n] = 1.0;
                    } else if (nfull == 0) {
                        flag[n] = 0;
                        cvof[n] = 0.0;
                    } else {
                        flag[n] = 2;
                    }
                }
            }
}

/* levelset2vof(shapes2ls, 0) without VOFI (vofmodules.f90:1048-1109) followed by
 * the end of initconditions_VOF (:788-792): ghosts, SetVOFBC, phase. */
static int og_init_shapes_impl(const paris_grid_desc* desc, int nb, const double* xc, const double* yc,
                               const double* zc, const double* rad, const double* excentricity, int ipar,
                               int refinement, int jacobi, double* cvof, int32_t* flag, int32_t* phase);

int og_init_spheres(const paris_grid_desc* desc, int nb, const double* xc, const double* yc,
                    const double* zc, const double* rad, int refinement, int jacobi,
                    double* cvof, int32_t* flag, int32_t* phase) {
    return og_init_shapes_impl(desc, nb, xc, yc, zc, rad, NULL, 0, refinement, jacobi, cvof, flag, phase);
}

/* levelset2vof(shapes2ls, ipar) with the excentricity of module_2phase:
 * ipar = 0 spheres, -1/-2/-3 a cylinder along x/y/z (one bubble). */
int og_init_shapes(const paris_grid_desc* desc, int nb, const double* xc, const double* yc, const double* zc,
                   const double* rad, const double* excentricity, int ipar, int refinement, double* cvof,
                   int32_t* flag, int32_t* phase) {
    if (ipar < -3 || ipar > 0 || (ipar < 0 && nb != 1)) return PARIS_BAD_ARGS;
    return og_init_shapes_impl(desc, nb, xc, yc, zc, rad, excentricity, ipar, refinement, 0, cvof, flag, phase);
}

static int og_levelset2vof(og_grid* g, og_spheres* s, int refinement, int jacobi, double* cvof, int32_t* flag,
                           int32_t* phase);

/* levelset2vof(wave2ls, ipar) (vofmodules.f90:683-689, 997-1034): ipar 1, 2
 * or 3 puts the interface normal to z, z or y and varying along y, x, x;
 * A_h = 2, normal_up and hshift as in the reference's namelist. */
int og_init_wave(const paris_grid_desc* desc, int ipar, int normal_up, double hshift, int refinement, double* cvof,
                 int32_t* flag, int32_t* phase) {
    if (ipar < 1 || ipar > 3) return PARIS_BAD_ARGS;
    og_grid* g = og_grid_new(desc);
    og_spheres s;
    memset(&s, 0, sizeof(s));
    s.wave = 1;
    const int hpar = ipar == 1 ? 2 : 1, vpar = ipar == 3 ? 2 : 3;   /* 1-based */
    for (int a = 0; a < 3; a++) {
        s.hdir[a] = a + 1 == hpar ? 1.0 : 0.0;
        s.vdir[a] = a + 1 == vpar ? 1.0 : 0.0;
    }
    s.len[0] = desc->xlength; s.len[1] = desc->ylength; s.len[2] = desc->zlength;
    const double A_h = 2.0;
    const double dxm = g->dx[g->nx / 2 + 2 - 1];   /* dx(nx/2+2) */
    s.amp = 0.5 * A_h * dxm;
    s.nsign = normal_up ? 1.0 : -1.0;
    s.shift = hshift * dxm;
    return og_levelset2vof(g, &s, refinement, 0, cvof, flag, phase);
}

static int og_init_shapes_impl(const paris_grid_desc* desc, int nb, const double* xc, const double* yc,
                               const double* zc, const double* rad, const double* excentricity, int ipar,
                               int refinement, int jacobi, double* cvof, int32_t* flag, int32_t* phase) {
    og_grid* g = og_grid_new(desc);
    og_spheres s;
    s.nb = nb; s.xc = xc; s.yc = yc; s.zc = zc; s.rad = rad; s.ncand = 0;
    s.wave = 0;
    for (int a = 0; a < 3; a++) s.cdir[a] = 1.0 / (1.0 + (excentricity ? excentricity[a] : 0.0));
    if (ipar < 0) s.cdir[-ipar - 1] = 0.0;
    s.prune = s.cdir[0] == 1.0 && s.cdir[1] == 1.0 && s.cdir[2] == 1.0;
    if (!s.prune) {
        s.ncand = nb < 4096 ? nb : 4096;
        for (int q = 0; q < s.ncand; q++) s.cand[q] = q;
    }
    return og_levelset2vof(g, &s, refinement, jacobi, cvof, flag, phase);
}

/* levelset2vof without VOFI (vofmodules.f90:1048-1109) followed by the end of
 * initconditions_VOF (:788-792): a first pass at refinement 1, ghosts and
 * SetVOFBC, the refined pass, ghosts, SetVOFBC, phase.  Frees g. */
static int og_levelset2vof(og_grid* g, og_spheres* sp, int refinement, int jacobi, double* cvof, int32_t* flag,
                           int32_t* phase) {
    og_spheres s = *sp;
    /* initialize_VOF: cvof = 0, vof_flag = 3 (vofmodules.f90:436-437) */
    for (long n = 0; n < g->ntot; n++) { cvof[n] = 0.0; flag[n] = 3; }
    og_ls2vof_refined(g, &s, 1, cvof, flag, flag);
    og_do_all_ighost(g, flag);
    og_do_all_ghost(g, cvof);
    og_setvofbc(g, cvof, flag);
    /* the second pass stops with "bad flag" unless the largest flag is 2
     * (vofmodules.f90:1220-1231); a 'jet' or '90deg' face leaves its second
     * ghost layer at 3 */
    int32_t fmax = -2147483647;
    for (long n = 0; n < g->ntot; n++) fmax = flag[n] > fmax ? flag[n] : fmax;
    if (refinement > 1 && fmax != 2) { og_grid_free(g); return PARIS_BAD_ARGS; }
    /* jacobi = 1: pass 2 reads the flags of pass 1 only (the order-free variant
     * computed by the device); 0: the reference's in-place loop order. */
    int32_t* f1 = NULL;
    if (jacobi) {
        f1 = malloc(g->ntot * sizeof(int32_t));
        memcpy(f1, flag, g->ntot * sizeof(int32_t));
    }
    og_ls2vof_refined(g, &s, refinement, cvof, flag, jacobi ? f1 : flag);
    free(f1);
    og_do_all_ghost(g, cvof);
    og_do_all_ighost(g, flag);
    og_setvofbc(g, cvof, flag);
    if (phase) og_vof_phase(g, cvof, phase);
    og_grid_free(g);
    return 0;
}

/* SetVOFBC on host arrays, for the tests */
int og_setvofbc_host(const paris_grid_desc* desc, double* cv, int32_t* fl) {
    og_grid* g = og_grid_new(desc);
    og_setvofbc(g, cv, fl);
    og_grid_free(g);
    return 0;
}
