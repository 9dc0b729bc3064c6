/*
 * og_st.c -- oracle (test infrastructure only): height functions, curvature
 * and the CSF surface force, restated from surface_tension.f90 and
 * paris.f90:2862-2957 in the same operation order.  Index arithmetic that
 * enters floating-point expressions uses the Fortran index values
 * (C index + 1), as the reference does.
 */
#include <math.h>
#include <string.h>
#include "og.h"

#define NDEPTH 3
#define BIGINT 100
#define D_HALF_BIGINT 50.0
#define UNCOMPUTED 2e6
#define NPOS 28
#define KAPPAMAX 4.0
#define NFOUND_MIN 6
#define EPS_GEOM 1e-4
#define TINYV 1e-50
#define UNDECIDED 5
#define UNCOMPUTABLE 4

typedef struct {
    const og_grid* g;
    const double* c;
    const int32_t* f;
    double* H;   /* 6 ghosted arrays */
    double epsc;
    int do_rotation, use_full_heights;
} og_st;

static inline double* HI(const og_st* s, int index1) { return s->H + (long)(index1 - 1) * s->g->ntot; }

static int coordlimit(const og_grid* g, int d, int sign) { return sign < 0 ? g->ng : g->ng + g->N[d] - 1; }

/* get_heights_pass1, surface_tension.f90:266-371 */
static void heights_pass1(og_st* s, int d) {
    const og_grid* g = s->g;
    long st[3] = {1, g->sy, g->sz};
    int ng = g->ng;
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                int f = s->f[n];
                if (f / 2 != 0) continue;
                for (int sign = -1; sign <= 1; sign += 2) {
                    int c[3] = {i, j, k};
                    int normalsign = (2 * f - 1) * sign;
                    int index = 2 * d + 1 + (-normalsign + 1) / 2;
                    double* H = HI(s, index);
                    int other = 1 - f;
                    int climitp1 = coordlimit(g, d, sign) + sign;
                    double hp = 0.0;
                    int sstep = 0, c0 = c[d], c1 = c0 + sign * NDEPTH;
                    int abandon = 0;
                    int found_at_start = H[n] < D_HALF_BIGINT;
                    while (!abandon) {
                        long cc = c[0] + c[1] * st[1] + c[2] * st[2];
                        int same = sstep > 0 && s->f[cc] == f;
                        hp = hp + (s->c[cc] - 0.5) * normalsign;
                        abandon = same || found_at_start || s->f[cc] == other || c[d] == climitp1 ||
                                  sstep == 2 * NDEPTH;
                        if (!abandon) {
                            sstep++;
                            c[d] += sign;
                        } else if (s->f[cc] == other) {
                            hp = hp + (2 * NDEPTH - sstep) * (s->c[cc] - 0.5) * normalsign;
                            while (c[d] != c0 - sign) {
                                long q = c[0] + c[1] * st[1] + c[2] * st[2];
                                H[q] = hp + (double)(c1 + 1) - (double)(c[d] + 1);
                                c[d] -= sign;
                            }
                        } else if (c[d] == climitp1) {
                            hp = hp + (-s->c[cc] + 0.5) * normalsign;
                            c[d] -= sign;
                            long q = c[0] + c[1] * st[1] + c[2] * st[2];
                            H[q] = hp + (double)(BIGINT * sstep);
                        }
                    }
                }
            }
}

/* get_heights_pass2, surface_tension.f90:375-448 */
static void heights_pass2(og_st* s, int d) {
    const og_grid* g = s->g;
    long st[3] = {1, g->sy, g->sz};
    int t2 = (d + 1) % 3, t3 = (d + 2) % 3;
    if (t2 > t3) { int t = t2; t2 = t3; t3 = t; }
    int ng = g->ng;
    for (int l = ng; l < ng + g->N[t2]; l++)
        for (int m = ng; m < ng + g->N[t3]; m++) {
            int c[3];
            c[t2] = l; c[t3] = m;
            for (int sign = -1; sign <= 1; sign += 2)
                for (int index = 2 * d + 1; index <= 2 * d + 2; index++) {
                    double* H = HI(s, index);
                    int cb = coordlimit(g, d, sign);
                    c[d] = cb;
                    double hb = H[c[0] + c[1] * st[1] + c[2] * st[2]];
                    if (hb > D_HALF_BIGINT && hb < 1e6) {
                        c[d] = cb + sign;
                        double ha = H[c[0] + c[1] * st[1] + c[2] * st[2]];
                        c[d] = cb;
                        if (ha < D_HALF_BIGINT) {
                            H[c[0] + c[1] * st[1] + c[2] * st[2]] = ha + sign;
                        } else if (ha > D_HALF_BIGINT && ha < 1e6) {
                            int sbelow = (int)floorf((float)(hb + D_HALF_BIGINT) / (float)BIGINT);
                            hb = hb - BIGINT * sbelow;
                            int sabove = (int)floorf((float)(ha + D_HALF_BIGINT) / (float)BIGINT);
                            ha = ha - BIGINT * sabove;
                            if (sabove + sbelow - 1 <= 2 * NDEPTH + 1) {
                                int c0 = cb - (sbelow - 1) * sign;
                                double cmiddle = (double)(c0 + 1) + sign * (sabove + sbelow - 1) * 0.5;
                                c[d] = cb + 2 * sign;
                                while (c[d] != c0 - sign) {
                                    H[c[0] + c[1] * st[1] + c[2] * st[2]] = ha + hb + cmiddle - (double)(c[d] + 1);
                                    c[d] -= sign;
                                }
                            }
                        }
                    }
                }
        }
    for (int index = 2 * d + 1; index <= 2 * d + 2; index++) {
        double* H = HI(s, index);
        for (long q = 0; q < g->ntot; q++)
            if (H[q] > D_HALF_BIGINT) H[q] = 2e6;
    }
}

/* get_all_heights, surface_tension.f90:185-260.  H: 6 ghosted arrays. */
int og_get_all_heights(const paris_grid_desc* desc, const double* cvof, const int32_t* flag, double* H) {
    og_grid* g = og_grid_new(desc);
    og_st s = {g, cvof, flag, H, desc->epsc, desc->do_rotation, desc->use_full_heights};
    for (long q = 0; q < 6 * g->ntot; q++) H[q] = 2e6;
    for (int d = 0; d < 3; d++) heights_pass1(&s, d);
    for (int q = 0; q < 6; q++) og_do_all_ghost(g, H + q * g->ntot);
    for (int d = 0; d < 3; d++) heights_pass2(&s, d);
    for (int q = 0; q < 6; q++) og_do_all_ghost(g, H + q * g->ntot);
    og_grid_free(g);
    return 0;
}

/* ---- curvature --------------------------------------------------------- */

/* orientation: indices sorted by |m| descending (bubble sort),
 * surface_tension.f90:1584-1601 (0-based here) */
static void og_orientation(const double m[3], int c[3]) {
    c[0] = 0; c[1] = 1; c[2] = 2;
    for (int i = 1; i <= 2; i++)
        for (int j = 1; j <= 3 - i; j++)
            if (fabs(m[c[j]]) > fabs(m[c[j - 1]])) {
                int t = c[j - 1]; c[j - 1] = c[j]; c[j] = t;
            }
}

static void og_threshold(double* z) {
    if (*z < 0.0) *z = 0.0;
    else if (*z > 1.0) *z = 1.0;
}

/* LineCenter, surface_tension.f90:1532-1580 */
static void og_line_center(double dmx, double dmy, double alpha, double* px, double* py) {
    if (dmx < EPS_GEOM) { *px = 0.5; *py = alpha; return; }
    if (dmy < EPS_GEOM) { *py = 0.5; *px = alpha; return; }
    *px = 0.; *py = 0.0;
    if (alpha >= dmx) { *px = *px + 1.0; *py = *py + (alpha - dmx) / dmy; }
    else { *px = *px + alpha / dmx; }
    if (alpha >= dmy) { *py = *py + 1.0; *px = *px + (alpha - dmy) / dmx; }
    else { *py = *py + alpha / dmy; }
    *px = *px / 2.0;
    *py = *py / 2.0;
    og_threshold(px);
    og_threshold(py);
}

/* PlaneAreaCenter, surface_tension.f90:1421-1529 (the argument checks of the
 * reference abort; here they cannot trigger for normals from youngs) */
static void og_plane_area_center(double dmx, double dmy, double dmz, double alpha, double* px, double* py, double* pz) {
    double nx, ny, qx, qy, area, b, amax;
    if (dmx < EPS_GEOM) {
        nx = dmy; ny = dmz;
        og_line_center(nx, ny, alpha, &qx, &qy);
        *px = 0.5; *py = qx; *pz = qy;
        return;
    }
    if (dmy < EPS_GEOM) {
        nx = dmz; ny = dmx;
        og_line_center(nx, ny, alpha, &qx, &qy);
        *px = qy; *py = 0.5; *pz = qx;
        return;
    }
    if (dmz < EPS_GEOM) {
        og_line_center(dmx, dmy, alpha, px, py);
        *pz = 0.5;
        return;
    }
    if (alpha < EPS_GEOM) { *px = 0.0; *py = 0.0; *pz = 0.0; return; }
    if (alpha > 1.0 - EPS_GEOM) { *px = 1.0; *py = 1.0; *pz = 1.0; return; }
    area = alpha * alpha;
    *px = area * alpha; *py = area * alpha; *pz = area * alpha;
    b = alpha - dmx;
    if (b > 0.) { area = area - b * b; *px = *px - b * b * (2.0 * dmx + alpha); *py = *py - b * b * b; *pz = *pz - b * b * b; }
    b = alpha - dmy;
    if (b > 0.0) { area = area - b * b; *py = *py - b * b * (2.0 * dmy + alpha); *px = *px - b * b * b; *pz = *pz - b * b * b; }
    b = alpha - dmz;
    if (b > 0.0) { area = area - b * b; *pz = *pz - b * b * (2.0 * dmz + alpha); *px = *px - b * b * b; *py = *py - b * b * b; }
    amax = alpha - 1.0;
    b = amax + dmx;
    if (b > 0.0) {
        area = area + b * b;
        *py = *py + b * b * (2.0 * dmy + alpha - dmz);
        *pz = *pz + b * b * (2.0 * dmz + alpha - dmy);
        *px = *px + b * b * b;
    }
    b = amax + dmy;
    if (b > 0.0) {
        area = area + b * b;
        *px = *px + b * b * (2.0 * dmx + alpha - dmz);
        *pz = *pz + b * b * (2.0 * dmz + alpha - dmx);
        *py = *py + b * b * b;
    }
    b = amax + dmz;
    if (b > 0.0) {
        area = area + b * b;
        *px = *px + b * b * (2.0 * dmx + alpha - dmy);
        *py = *py + b * b * (2.0 * dmy + alpha - dmx);
        *pz = *pz + b * b * b;
    }
    area = 3.0 * area;
    *px = *px / (area * dmx);
    *py = *py / (area * dmy);
    *pz = *pz / (area * dmz);
    og_threshold(px);
    og_threshold(py);
    og_threshold(pz);
}

static void og_block(const og_st* s, long n, double st[27]) {
    const og_grid* g = s->g;
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int e = -1; e <= 1; e++) st[OG_C3(a + 1, b + 1, e + 1)] = s->c[n + a + b * g->sy + e * g->sz];
}

/* FindCutAreaCentroid, surface_tension.f90:1341-1409 */
static void og_find_cut_area_centroid(const og_st* s, long n, double cen[3]) {
    double st[27], nr[3];
    og_block(s, n, st);
    og_youngs(st, nr);
    double dmx = nr[0], dmy = nr[1], dmz = nr[2];
    double invx = 1.0, invy = 1.0, invz = 1.0;
    if (dmx < 0.0) { dmx = -dmx; invx = -1.0; }
    if (dmy < 0.0) { dmy = -dmy; invy = -1.0; }
    if (dmz < 0.0) { dmz = -dmz; invz = -1.0; }
    double m[3] = {dmx, dmy, dmz};
    double alpha = og_al3d(m, s->c[n]);
    double px, py, pz;
    og_plane_area_center(dmx, dmy, dmz, alpha, &px, &py, &pz);
    cen[0] = px * invx; cen[1] = py * invy; cen[2] = pz * invz;
    cen[0] = cen[0] - invx * 0.5;
    cen[1] = cen[1] - invy * 0.5;
    cen[2] = cen[2] - invz * 0.5;
}

/* NewFindCutAreaCentroid, surface_tension.f90:1316-1338 */
static void og_new_find_cut_area_centroid(const og_st* s, long n, double cen[3]) {
    double st[27], nr[3];
    og_block(s, n, st);
    og_youngs(st, nr);
    og_area_centroid(nr, s->c[n], cen);
    cen[0] = cen[0] - 0.5; cen[1] = cen[1] - 0.5; cen[2] = cen[2] - 0.5;
}

/* FindInverseMatrix, surface_tension.f90:1225-1313 (n = 6) */
static int og_find_inverse(const double mat[6][6], double inv[6][6], double epsc) {
    const int n = 6;
    double aug[6][12];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 2 * n; j++) {
            if (j < n) aug[i][j] = mat[i][j];
            else if (i + n == j) aug[i][j] = 1.0;
            else aug[i][j] = 0.0;
        }
    for (int k = 0; k < n - 1; k++)
        if (fabs(aug[k][k]) < epsc)
            for (int i = k + 1; i < n; i++)
                if (fabs(aug[i][k]) > epsc)
                    for (int l = 0; l < 2 * n; l++) aug[k][l] = aug[k][l] + aug[i][l];
    for (int k = 0; k < n - 1; k++) {
        if (fabs(aug[k][k]) < epsc) return 0;
        for (int j = k + 1; j < n; j++) {
            double m = aug[j][k] / aug[k][k];
            for (int i = k; i < 2 * n; i++) aug[j][i] = aug[j][i] - m * aug[k][i];
        }
    }
    if (fabs(aug[n - 1][n - 1]) < epsc) return 0;
    for (int i = 0; i < n; i++) {
        double m = aug[i][i];
        for (int j = i; j < 2 * n; j++) aug[i][j] = aug[i][j] / m;
    }
    for (int k = n - 2; k >= 0; k--)
        for (int i = 0; i <= k; i++) {
            double m = aug[i][k + 1];
            for (int j = k; j < 2 * n; j++) aug[i][j] = aug[i][j] - aug[k + 1][j] * m;
        }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) inv[i][j] = aug[i][n + j];
    return 1;
}

/* parabola_fit, surface_tension.f90:1136-1216; fit[q][0..2] */
static int og_parabola_fit(double fit[NPOS][3], const double w[NPOS], int np, double a[6], double epsc) {
    double m[6][6], inv[6][6], rhs[6];
    memset(m, 0, sizeof(m));
    memset(rhs, 0, sizeof(rhs));
    for (int q = 0; q < 6; q++) a[q] = 0.0;
    for (int f = 0; f < np; f++) {
        double x1 = fit[f][0], x2 = x1 * fit[f][0], x3 = x2 * fit[f][0], x4 = x3 * fit[f][0];
        double y1 = fit[f][1], y2 = y1 * fit[f][1], y3 = y2 * fit[f][1], y4 = y3 * fit[f][1];
        double wg = w[f];
        m[0][0] = m[0][0] + x4 * wg;
        m[1][1] = m[1][1] + y4 * wg;
        m[2][2] = m[2][2] + x2 * y2 * wg;
        m[3][3] = m[3][3] + x2 * wg;
        m[4][4] = m[4][4] + y2 * wg;
        m[5][5] = m[5][5] + wg;
        m[0][2] = m[0][2] + x3 * y1 * wg;
        m[0][3] = m[0][3] + x3 * wg;
        m[0][4] = m[0][4] + x2 * y1 * wg;
        m[1][2] = m[1][2] + x1 * y3 * wg;
        m[1][3] = m[1][3] + x1 * y2 * wg;
        m[1][4] = m[1][4] + y3 * wg;
        m[2][5] = m[2][5] + x1 * y1 * wg;
        m[3][5] = m[3][5] + x1 * wg;
        m[4][5] = m[4][5] + y1 * wg;
        rhs[0] = rhs[0] + x2 * fit[f][2] * wg;
        rhs[1] = rhs[1] + y2 * fit[f][2] * wg;
        rhs[2] = rhs[2] + x1 * y1 * fit[f][2] * wg;
        rhs[3] = rhs[3] + x1 * fit[f][2] * wg;
        rhs[4] = rhs[4] + y1 * fit[f][2] * wg;
        rhs[5] = rhs[5] + fit[f][2] * wg;
    }
    m[0][1] = m[2][2];
    m[0][5] = m[3][3];
    m[1][5] = m[4][4];
    m[2][3] = m[0][4];
    m[2][4] = m[1][3];
    m[3][4] = m[2][5];
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++)
            if (i > j) m[i][j] = m[j][i];
    if (!og_find_inverse(m, inv, epsc)) return 0;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) a[i] = a[i] + inv[i][j] * rhs[j];
    return 1;
}

/* parabola_fit_with_rotation, surface_tension.f90:1056-1129 */
static int og_parabola_fit_rot(const og_st* s, double bfit[NPOS][3], const double w[NPOS], const double mv[3],
                               int np, double a[6], double* ksign) {
    if (s->do_rotation) {
        double ev[3][3], nrm[3], fit[NPOS][3];
        ev[0][2] = mv[0]; ev[1][2] = mv[1]; ev[2][2] = mv[2];
        *ksign = 1.0;
        ev[0][0] = mv[2];
        ev[1][0] = 0.0;
        ev[2][0] = -mv[0];
        ev[0][1] = -ev[1][0] * ev[2][2] + ev[2][0] * ev[1][2];
        ev[1][1] = ev[0][0] * ev[2][2] - ev[2][0] * ev[0][2];
        ev[2][1] = -ev[0][0] * ev[1][2] + ev[1][0] * ev[0][2];
        for (int c = 0; c < 3; c++) nrm[c] = sqrt(ev[0][c] * ev[0][c] + ev[1][c] * ev[1][c] + ev[2][c] * ev[2][c]);
        for (int i = 0; i < 3; i++)
            for (int c = 0; c < 3; c++) ev[i][c] = ev[i][c] / nrm[c];
        memcpy(fit, bfit, sizeof(fit));
        for (int i = 0; i < 3; i++)
            for (int q = 0; q < NPOS; q++) bfit[q][i] = ev[0][i] * fit[q][0] + ev[1][i] * fit[q][1] + ev[2][i] * fit[q][2];
    } else {
        *ksign = copysign(1.0, mv[2]);
    }
    return og_parabola_fit(bfit, w, np, a, s->epsc);
}

/* ind_pos_sorted_add, surface_tension.f90:1667-1702 */
static int og_ind_pos_sorted_add(const double cen[3], double pts[NPOS][3], double bp[NPOS][3], int n) {
    bp[0][0] = cen[0]; bp[0][1] = cen[1]; bp[0][2] = cen[2];
    if (n < 2) return n;
    int ni = 2;
    bp[1][0] = pts[0][0]; bp[1][1] = pts[0][1]; bp[1][2] = pts[0][2];
    for (int j = 1; j < n; j++) {
        int reject = 0;
        for (int i = 0; i < j; i++)
            if (!reject) {
                double d2 = 0.0;
                for (int c = 0; c < 3; c++) {
                    double t = pts[i][c] - pts[j][c];
                    d2 = d2 + t * t;
                }
                reject = d2 < 0.5 * 0.5;
            }
        if (!reject) {
            ni++;
            bp[ni - 1][0] = pts[j][0]; bp[ni - 1][1] = pts[j][1]; bp[ni - 1][2] = pts[j][2];
        }
    }
    return ni;
}

/* map3x3in2x2 (vofmodules.f90:1172-1193) position (m,n) of the 3x3 plane
 * normal to d around (i0,j0,k0) */
static void og_map(int d, int m, int nn, int i0, int j0, int k0, int p[3]) {
    if (d == 0) { p[0] = i0; p[1] = m + j0; p[2] = nn + k0; }
    else if (d == 1) { p[0] = m + i0; p[1] = j0; p[2] = nn + k0; }
    else { p[0] = m + i0; p[1] = nn + j0; p[2] = k0; }
}

/* get_local_heights, surface_tension.f90:490-589.  try[] 0-based; h[m+1][n+1]. */
static int og_get_local_heights(const og_st* s, int i, int j, int k, const double mxyz[3], int try_[3],
                                double h[3][3], double pts[NPOS][3], int* nposit) {
    const og_grid* g = s->g;
    int nfound = 0;
    memset(pts, 0, sizeof(double) * NPOS * 3);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) h[a][b] = 2e6;
    *nposit = 0;
    for (int l = 0; l < 3; l++) {
        int d = try_[l];
        int si = d == 0, sj = d == 1, sk = d == 2;
        int index = 2 * d + 2;
        if (mxyz[d] > 0) index = 2 * d + 1;
        const double* H = HI(s, index);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) h[a][b] = 2e6;
        nfound = 0;
        for (int m = -1; m <= 1; m++)
            for (int nn = -1; nn <= 1; nn++) {
                int p[3];
                og_map(d, m, nn, i, j, k, p);
                double hv = H[OG_IX(g, p[0], p[1], p[2])];
                int got = 0;
                if (hv < 1e6) {
                    h[m + 1][nn + 1] = hv;
                    got = 1;
                } else {
                    for (int st = 1; st <= g->ng && !got; st++) {
                        double hu = H[OG_IX(g, p[0] + si * st, p[1] + sj * st, p[2] + sk * st)];
                        double hd = H[OG_IX(g, p[0] - si * st, p[1] - sj * st, p[2] - sk * st)];
                        if (hu < 1e6) { h[m + 1][nn + 1] = hu + st; got = 1; }
                        else if (hd < 1e6) { h[m + 1][nn + 1] = hd - st; got = 1; }
                    }
                }
                if (got) {
                    nfound++;
                    int q = (*nposit)++;
                    double hl = h[m + 1][nn + 1];
                    pts[q][0] = hl * si + (double)(p[0] + 1) - (double)(i + 1);
                    pts[q][1] = hl * sj + (double)(p[1] + 1) - (double)(j + 1);
                    pts[q][2] = hl * sk + (double)(p[2] + 1) - (double)(k + 1);
                }
            }
        if (nfound == 9) {
            int t[3], nn = 1;
            for (int m = 0; m < 3; m++)
                if (m != d) t[nn++] = m;
            t[0] = d;
            try_[0] = t[0]; try_[1] = t[1]; try_[2] = t[2];
            return 9;
        }
    }
    return nfound;
}

/* curvature_pop_pass1, surface_tension.f90:827-932 */
static double og_curv_pass1(const og_st* s, int i0, int j0, int k0, int* nfound_out) {
    const og_grid* g = s->g;
    long n = OG_IX(g, i0, j0, k0);
    double st[27], mxyz[3], h[3][3], pts[NPOS][3], bp[NPOS][3], origin[3], mv[3], a[6], w[NPOS];
    int try_[3], nposit;
    double kappa = UNCOMPUTED;
    og_block(s, n, st);
    og_mycs(st, mxyz);
    og_orientation(mxyz, try_);
    int nfound = og_get_local_heights(s, i0, j0, k0, mxyz, try_, h, pts, &nposit);
    if (fabs(mxyz[0]) < TINYV && fabs(mxyz[1]) < TINYV && fabs(mxyz[2]) < TINYV) {
        *nfound_out = 21;
        return kappa;
    }
    if (nfound == 9 && s->use_full_heights) {
        double a1 = h[2][1] - 2.0 * h[1][1] + h[0][1];
        double a2 = h[1][2] - 2.0 * h[1][1] + h[1][0];
        double a3 = (h[2][2] - h[0][2] - h[2][0] + h[0][0]) / 4.0;
        double a4 = (h[2][1] - h[0][1]) / 2.0;
        double a5 = (h[1][2] - h[1][0]) / 2.0;
        kappa = (a1 * (1.0 + a5 * a5) + a2 * (1.0 + a4 * a4) - 2.0 * a3 * a4 * a5) /
                pow(1.0 + a4 * a4 + a5 * a5, 1.5);
        kappa = copysign(1.0, mxyz[try_[0]]) * kappa;
        *nfound_out = 0;
        return kappa;
    }
    og_find_cut_area_centroid(s, n, origin);
    nfound = og_ind_pos_sorted_add(origin, pts, bp, nposit);
    mv[0] = mxyz[try_[1]]; mv[1] = mxyz[try_[2]]; mv[2] = mxyz[try_[0]];
    if (nfound > NFOUND_MIN + 1) {
        double p2[NPOS][3];
        for (int q = 0; q < nfound; q++) {
            p2[q][0] = bp[q][try_[1]] - origin[try_[1]];
            p2[q][1] = bp[q][try_[2]] - origin[try_[2]];
            p2[q][2] = bp[q][try_[0]] - origin[try_[0]];
        }
        for (int q = nfound; q < NPOS; q++) p2[q][0] = p2[q][1] = p2[q][2] = 0.0;
        for (int q = 0; q < NPOS; q++) w[q] = 1.0;
        w[0] = 1e2 * og_area3d(mxyz, s->c[n]);
        double ks;
        if (og_parabola_fit_rot(s, p2, w, mv, nfound, a, &ks)) {
            kappa = 2.0 * (a[0] * (1.0 + a[4] * a[4]) + a[1] * (1.0 + a[3] * a[3]) - a[2] * a[3] * a[4]) /
                    pow(1.0 + a[3] * a[3] + a[4] * a[4], 1.5);
            kappa = ks * kappa;
            *nfound_out = -nfound;
            return kappa;
        }
        *nfound_out = 16;
        return kappa;
    }
    *nfound_out = nfound + 1;
    return kappa;
}

/* curvature_pop_pass2, surface_tension.f90:959-1052 */
static double og_curv_pass2(const og_st* s, int i0, int j0, int k0, int* nfound_out) {
    const og_grid* g = s->g;
    long n = OG_IX(g, i0, j0, k0);
    double st[27], mxyz[3], origin[3], mv[3], a[6], w[NPOS], fit[NPOS][3], pts[NPOS][3];
    int try_[3];
    double kappa = UNCOMPUTED;
    og_block(s, n, st);
    og_fd32(st, mxyz);
    og_orientation(mxyz, try_);
    if (fabs(mxyz[0]) < TINYV && fabs(mxyz[1]) < TINYV && fabs(mxyz[2]) < TINYV) {
        *nfound_out = 21;
        return kappa;
    }
    og_find_cut_area_centroid(s, n, origin);
    mv[0] = mxyz[try_[1]]; mv[1] = mxyz[try_[2]]; mv[2] = mxyz[try_[0]];
    int nposit = 0;
    for (int m = -1; m <= 1; m++)
        for (int nn = -1; nn <= 1; nn++)
            for (int l = -1; l <= 1; l++) {
                long q = OG_IX(g, i0 + m, j0 + nn, k0 + l);
                double wg = s->c[q] * (1.0 - s->c[q]);
                if (s->f[q] == 2 && wg > 0.0) {
                    double cen[3];
                    og_new_find_cut_area_centroid(s, q, cen);
                    fit[nposit][0] = cen[0] + m;
                    fit[nposit][1] = cen[1] + nn;
                    fit[nposit][2] = cen[2] + l;
                    w[nposit] = 1.0;
                    nposit++;
                }
            }
    for (int q = 0; q < nposit; q++) {
        pts[q][0] = fit[q][try_[1]] - origin[try_[1]];
        pts[q][1] = fit[q][try_[2]] - origin[try_[2]];
        pts[q][2] = fit[q][try_[0]] - origin[try_[0]];
    }
    for (int q = nposit; q < NPOS; q++) { pts[q][0] = pts[q][1] = pts[q][2] = 0.0; w[q] = 1.0; }
    if (nposit < 6) {
        *nfound_out = nposit + 10;
        return kappa;
    }
    double ks;
    if (!og_parabola_fit_rot(s, pts, w, mv, nposit, a, &ks)) {
        *nfound_out = 16;
        return kappa;
    }
    double sq = sqrt(1.0 + a[3] * a[3] + a[4] * a[4]);
    kappa = 2.0 * (a[0] * (1.0 + a[4] * a[4]) + a[1] * (1.0 + a[3] * a[3]) - a[2] * a[3] * a[4]) / (sq * sq * sq);
    kappa = ks * kappa;
    *nfound_out = -nposit - 50;
    return kappa;
}

/* get_all_curvatures_pop, surface_tension.f90:651-755.  H from
 * og_get_all_heights; kappa ghosted out; kflag (ghosted, optional) out. */
int og_get_all_curvatures(const paris_grid_desc* desc, const double* cvof, const int32_t* flag, const double* H,
                          double* kappa, int32_t* kflag_out, int32_t* method_count) {
    og_grid* g = og_grid_new(desc);
    og_st s = {g, cvof, flag, (double*)H, desc->epsc, desc->do_rotation, desc->use_full_heights};
    int32_t* kf = malloc(g->ntot * sizeof(int32_t));
    int mc[5] = {0, 0, 0, 0, 0};
    int ng = g->ng;
    for (long q = 0; q < g->ntot; q++) { kappa[q] = UNCOMPUTED; kf[q] = UNDECIDED; }
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                if (flag[n] != 2) continue;
                int nf;
                kappa[n] = og_curv_pass1(&s, i, j, k, &nf);
                if (nf == 0) { kf[n] = 0; mc[0]++; }
                if (nf > -50 && nf < 0) { kf[n] = 1; mc[1]++; }
            }
    og_do_all_ghost(g, kappa);
    og_do_all_ighost(g, kf);
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                if (flag[n] != 2 || kf[n] <= 1) continue;
                int cnt = 0;
                double kap = 0.0;
                for (int m = -1; m <= 1; m++)
                    for (int nn = -1; nn <= 1; nn++)
                        for (int l = -1; l <= 1; l++) {
                            long q = OG_IX(g, i + m, j + nn, k + l);
                            if (kf[q] < 2) { cnt++; kap = kap + kappa[q]; }
                        }
                if (cnt > 0) { kappa[n] = kap / cnt; kf[n] = 2; mc[2]++; }
            }
    for (int k = ng; k < ng + g->nz; k++)
        for (int j = ng; j < ng + g->ny; j++)
            for (int i = ng; i < ng + g->nx; i++) {
                long n = OG_IX(g, i, j, k);
                if (flag[n] == 2) {
                    if (kf[n] > 2) {
                        int nf;
                        double kap = og_curv_pass2(&s, i, j, k, &nf);
                        if (nf > 0) { kf[n] = UNCOMPUTABLE; mc[4]++; }
                        else { kappa[n] = kap; kf[n] = 3; mc[3]++; }
                    }
                } else {
                    kf[n] = UNCOMPUTABLE;
                }
            }
    og_do_all_ghost(g, kappa);
    og_do_all_ighost(g, kf);
    for (long q = 0; q < g->ntot; q++)
        if (kf[q] < UNCOMPUTABLE) {
            double kap = kappa[q];
            if (fabs(kap) > KAPPAMAX) kap = copysign(1.0, kap) * KAPPAMAX;
            kappa[q] = kap;
        }
    if (kflag_out) memcpy(kflag_out, kf, g->ntot * sizeof(int32_t));
    if (method_count) for (int q = 0; q < 5; q++) method_count[q] = mc[q];
    free(kf);
    og_grid_free(g);
    return 0;
}

/* surfaceForce, paris.f90:2862-2957 (du,dv,dw += CSF force; kappa ghosted) */
int og_surface_force(const paris_grid_desc* desc, const double* cvof, const double* kappa, const double* rho,
                     double* du, double* dv, double* dw) {
    og_grid* g = og_grid_new(desc);
    int ng = g->ng;
    double deltax = g->dx[g->nx - 1];   /* dx(nx) */
    double sigma = desc->sigma, epsc = desc->epsc;
    long st[3] = {1, g->sy, g->sz};
    double* out[3] = {du, dv, dw};
    const double* dh[3] = {g->dxh, g->dyh, g->dzh};
    for (int d = 0; d < 3; d++) {
        int lim = ng + g->N[d] - 1;   /* ieu = ie - 1 when not periodic */
        if (desc->bdry_cond[d] != PARIS_BC_PERIODIC) lim--;
        for (int k = ng; k < ng + g->nz; k++)
            for (int j = ng; j < ng + g->ny; j++)
                for (int i = ng; i < ng + g->nx; i++) {
                    int c[3] = {i, j, k};
                    if (c[d] > lim) continue;
                    long n = OG_IX(g, i, j, k), o = st[d];
                    if (fabs(cvof[n + o] - cvof[n]) > epsc / 1e1) {
                        int cnt = 0;
                        double kap = 0.0;
                        if (kappa[n + o] < 1e6) { kap = kap + kappa[n + o]; cnt++; }
                        if (kappa[n] < 1e6) { kap = kap + kappa[n]; cnt++; }
                        if (cnt > 0) {
                            kap = kap / (deltax * cnt);
                            out[d][n] = out[d][n] - kap * sigma * (2.0 / dh[d][c[d]]) * (cvof[n + o] - cvof[n]) /
                                                        (rho[n + o] + rho[n]);
                        }
                    }
                }
    }
    og_grid_free(g);
    return 0;
}
