/*
 * og_mom.c -- oracle of the explicit momentum predictor (test
 * infrastructure only): momentumConvectionQUICK (paris.f90:2288-2414),
 * momentumConvection_onedim with slope_lim (paris.f90:1991-2071,
 * modules.f90:177-197), explicitMomDiff (paris.f90:2757-2808), volumeForce
 * (paris.f90:2813-2860), the wall part of SetVelocityBC
 * (modules.f90:951-973, 1061-1105) followed by do_ghost_vector
 * (modules.f90:1628-1642), and u = u + dt*du (paris.f90:442-444).
 *
 * Arrays are ghosted, C index = Fortran index - 1 (interior [ng, ng+n)).
 * Expressions keep the Fortran operation order (x**2 is x*x; the Fortran
 * single-precision literals 0.5, 0.25, 1., 2. are exact).
 */
#include <math.h>
#include <string.h>

#include "og.h"

#define IX(i, j, k) OG_IX(g, i, j, k)

typedef struct {
    og_grid* g;
    int is, ie, js, je, ks, ke, ieu, jev, kew;
} mom_rng;

static void rng_init(mom_rng* r, og_grid* g) {
    r->g = g;
    r->is = g->ng; r->ie = g->ng + g->nx - 1;
    r->js = g->ng; r->je = g->ng + g->ny - 1;
    r->ks = g->ng; r->ke = g->ng + g->nz - 1;
    r->ieu = r->ie - (og_is_periodic(g, 0) ? 0 : 1);
    r->jev = r->je - (og_is_periodic(g, 1) ? 0 : 1);
    r->kew = r->ke - (og_is_periodic(g, 2) ? 0 : 1);
}

/* inter(x0,x1,x2,x,y0,y1,y2), paris.f90:2390-2411 (QUICK branch) */
static double inter(double x0, double x1, double x2, double x, double y0, double y1, double y2) {
    double xi = (x - x0) / (x1 - x0);
    double k = (x2 - x0) / (x1 - x0);
    double a = (y2 - k * k * y1 + (k * k - 1.0) * y0) / k / (1.0 - k);
    double b = (y2 - k * y1 + (k - 1.0) * y0) / k / (k - 1.0);
    return y0 + a * xi + b * (xi * xi);
}

/* momentumConvectionQUICK, paris.f90:2288-2389: du, dv, dw are assigned on
 * the updated faces; work holds 3 ghosted scratch arrays */
int og_momentum_convection_quick(const paris_grid_desc* desc, const double* u, const double* v, const double* w,
                                 double* du, double* dv, double* dw) {
    og_grid* g = og_grid_new(desc);
    mom_rng R;
    rng_init(&R, g);
    double* W1 = calloc(g->ntot, sizeof(double));
    double* W2 = calloc(g->ntot, sizeof(double));
    double* W3 = calloc(g->ntot, sizeof(double));
    const double *x = g->x, *xh = g->xh, *y = g->y, *yh = g->yh, *z = g->z, *zh = g->zh;
    const double *dx = g->dx, *dxh = g->dxh, *dy = g->dy, *dyh = g->dyh, *dz = g->dz, *dzh = g->dzh;
    /* u-velocity */
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ieu + 1; i++) {
        if (u[IX(i - 1, j, k)] + u[IX(i, j, k)] > 0.0)
            W1[IX(i, j, k)] = inter(xh[i - 1], xh[i], xh[i - 2], x[i], u[IX(i - 1, j, k)], u[IX(i, j, k)], u[IX(i - 2, j, k)]);
        else
            W1[IX(i, j, k)] = inter(xh[i], xh[i - 1], xh[i + 1], x[i], u[IX(i, j, k)], u[IX(i - 1, j, k)], u[IX(i + 1, j, k)]);
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js - 1; j <= R.je; j++) for (int i = R.is - 1; i <= R.ie; i++) {
        if (v[IX(i, j, k)] + v[IX(i + 1, j, k)] > 0.0)
            W2[IX(i, j, k)] = inter(y[j], y[j + 1], y[j - 1], yh[j], u[IX(i, j, k)], u[IX(i, j + 1, k)], u[IX(i, j - 1, k)]);
        else
            W2[IX(i, j, k)] = inter(y[j + 1], y[j], y[j + 2], yh[j], u[IX(i, j + 1, k)], u[IX(i, j, k)], u[IX(i, j + 2, k)]);
    }
    for (int k = R.ks - 1; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is - 1; i <= R.ie; i++) {
        if (w[IX(i, j, k)] + w[IX(i + 1, j, k)] > 0.0)
            W3[IX(i, j, k)] = inter(z[k], z[k + 1], z[k - 1], zh[k], u[IX(i, j, k)], u[IX(i, j, k + 1)], u[IX(i, j, k - 1)]);
        else
            W3[IX(i, j, k)] = inter(z[k + 1], z[k], z[k + 2], zh[k], u[IX(i, j, k + 1)], u[IX(i, j, k)], u[IX(i, j, k + 2)]);
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ieu; i++) {
        double a = W1[IX(i + 1, j, k)], b = W1[IX(i, j, k)];
        du[IX(i, j, k)] = -(a * a - b * b) / dxh[i]
            - 0.5 * ((v[IX(i, j, k)] + v[IX(i + 1, j, k)]) * W2[IX(i, j, k)] -
                     (v[IX(i, j - 1, k)] + v[IX(i + 1, j - 1, k)]) * W2[IX(i, j - 1, k)]) / dy[j]
            - 0.5 * ((w[IX(i, j, k)] + w[IX(i + 1, j, k)]) * W3[IX(i, j, k)] -
                     (w[IX(i, j, k - 1)] + w[IX(i + 1, j, k - 1)]) * W3[IX(i, j, k - 1)]) / dz[k];
    }
    /* v-velocity */
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.jev + 1; j++) for (int i = R.is; i <= R.ie; i++) {
        if (v[IX(i, j - 1, k)] + v[IX(i, j, k)] > 0.0)
            W2[IX(i, j, k)] = inter(yh[j - 1], yh[j], yh[j - 2], y[j], v[IX(i, j - 1, k)], v[IX(i, j, k)], v[IX(i, j - 2, k)]);
        else
            W2[IX(i, j, k)] = inter(yh[j], yh[j - 1], yh[j + 1], y[j], v[IX(i, j, k)], v[IX(i, j - 1, k)], v[IX(i, j + 1, k)]);
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js - 1; j <= R.je; j++) for (int i = R.is - 1; i <= R.ie; i++) {
        if (u[IX(i, j, k)] + u[IX(i, j + 1, k)] > 0.0)
            W1[IX(i, j, k)] = inter(x[i], x[i + 1], x[i - 1], xh[i], v[IX(i, j, k)], v[IX(i + 1, j, k)], v[IX(i - 1, j, k)]);
        else
            W1[IX(i, j, k)] = inter(x[i + 1], x[i], x[i + 2], xh[i], v[IX(i + 1, j, k)], v[IX(i, j, k)], v[IX(i + 2, j, k)]);
    }
    for (int k = R.ks - 1; k <= R.ke; k++) for (int j = R.js - 1; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        if (w[IX(i, j, k)] + w[IX(i, j + 1, k)] > 0.0)
            W3[IX(i, j, k)] = inter(z[k], z[k + 1], z[k - 1], zh[k], v[IX(i, j, k)], v[IX(i, j, k + 1)], v[IX(i, j, k - 1)]);
        else
            W3[IX(i, j, k)] = inter(z[k + 1], z[k], z[k + 2], zh[k], v[IX(i, j, k + 1)], v[IX(i, j, k)], v[IX(i, j, k + 2)]);
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.jev; j++) for (int i = R.is; i <= R.ie; i++) {
        double a = W2[IX(i, j + 1, k)], b = W2[IX(i, j, k)];
        dv[IX(i, j, k)] = -0.5 * ((u[IX(i, j, k)] + u[IX(i, j + 1, k)]) * W1[IX(i, j, k)] -
                                  (u[IX(i - 1, j, k)] + u[IX(i - 1, j + 1, k)]) * W1[IX(i - 1, j, k)]) / dx[i]
            - (a * a - b * b) / dyh[j]
            - 0.5 * ((w[IX(i, j, k)] + w[IX(i, j + 1, k)]) * W3[IX(i, j, k)] -
                     (w[IX(i, j, k - 1)] + w[IX(i, j + 1, k - 1)]) * W3[IX(i, j, k - 1)]) / dz[k];
    }
    /* w-velocity */
    for (int k = R.ks; k <= R.kew + 1; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        if (w[IX(i, j, k - 1)] + w[IX(i, j, k)] > 0.0)
            W3[IX(i, j, k)] = inter(zh[k - 1], zh[k], zh[k - 2], z[k], w[IX(i, j, k - 1)], w[IX(i, j, k)], w[IX(i, j, k - 2)]);
        else
            W3[IX(i, j, k)] = inter(zh[k], zh[k - 1], zh[k + 1], z[k], w[IX(i, j, k)], w[IX(i, j, k - 1)], w[IX(i, j, k + 1)]);
    }
    for (int k = R.ks - 1; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is - 1; i <= R.ie; i++) {
        if (u[IX(i, j, k)] + u[IX(i, j, k + 1)] > 0.0)
            W1[IX(i, j, k)] = inter(x[i], x[i + 1], x[i - 1], xh[i], w[IX(i, j, k)], w[IX(i + 1, j, k)], w[IX(i - 1, j, k)]);
        else
            W1[IX(i, j, k)] = inter(x[i + 1], x[i], x[i + 2], xh[i], w[IX(i + 1, j, k)], w[IX(i, j, k)], w[IX(i + 2, j, k)]);
    }
    for (int k = R.ks - 1; k <= R.ke; k++) for (int j = R.js - 1; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        if (v[IX(i, j, k)] + v[IX(i, j, k + 1)] > 0.0)
            W2[IX(i, j, k)] = inter(y[j], y[j + 1], y[j - 1], yh[j], w[IX(i, j, k)], w[IX(i, j + 1, k)], w[IX(i, j - 1, k)]);
        else
            W2[IX(i, j, k)] = inter(y[j + 1], y[j], y[j + 2], yh[j], w[IX(i, j + 1, k)], w[IX(i, j, k)], w[IX(i, j + 2, k)]);
    }
    for (int k = R.ks; k <= R.kew; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        double a = W3[IX(i, j, k + 1)], b = W3[IX(i, j, k)];
        dw[IX(i, j, k)] = -0.5 * ((u[IX(i, j, k)] + u[IX(i, j, k + 1)]) * W1[IX(i, j, k)] -
                                  (u[IX(i - 1, j, k)] + u[IX(i - 1, j, k + 1)]) * W1[IX(i - 1, j, k)]) / dx[i]
            - 0.5 * ((v[IX(i, j, k)] + v[IX(i, j, k + 1)]) * W2[IX(i, j, k)] -
                     (v[IX(i, j - 1, k)] + v[IX(i, j - 1, k + 1)]) * W2[IX(i, j - 1, k)]) / dy[j]
            - (a * a - b * b) / dzh[k];
    }
    free(W1); free(W2); free(W3);
    og_grid_free(g);
    return 0;
}

/* minabs / maxabs, paris.f90:3450-3475 */
static double minabs(double a, double b) { return fabs(a) < fabs(b) ? a : b; }
static double maxabs(double a, double b) { return fabs(a) > fabs(b) ? a : b; }

/* slope_lim, modules.f90:177-197; scheme 1 ENO, 2 Superbee, 3 WENO */
static double slope_lim(double v1, double v2, double v3, int scheme) {
    if (scheme == 2) {
        double a1 = minabs(v3 - v2, 2.0 * (v2 - v1));
        double a2 = minabs(2.0 * (v3 - v2), v2 - v1);
        return maxabs(a1, a2);
    } else if (scheme == 1) {
        return minabs(v3 - v2, v2 - v1);
    } else if (scheme == 3) {
        double d1 = v2 - v1, d2 = v3 - v2;
        double a1 = 1.0 / (d1 * d1 + 1.e-16);
        double a2 = 1.0 / (d2 * d2 + 1.e-16);
        double a = a1 + a2;
        return (a1 * (v2 - v1) + a2 * (v3 - v2)) / a;
    }
    return 0.0;
}

/* momentumConvection_onedim, paris.f90:1991-2071, for direction d (1..3)
 * with phi the d-th velocity component; dphi assigned on its faces */
static void conv_onedim(og_grid* g, const mom_rng* R, const double* u, const double* v, const double* w,
                        const double* phi, double* dphi, int d, int scheme, double* W1, double* W2, double* W3) {
    int i0 = d == 1, j0 = d == 2, k0 = d == 3;
    int is0[3] = {R->is - 1, R->js - 1, R->ks - 1};
    int ie0[3] = {R->ie, R->je, R->ke};
    int is1[3], ie1[3];
    const double *dx = g->dx, *dy = g->dy, *dz = g->dz;
#define SETR(dd, top)                                   \
    for (int q = 0; q < 3; q++) { is1[q] = is0[q]; ie1[q] = ie0[q]; } \
    if (d == dd) { for (int q = 0; q < 3; q++) is1[q] += 1; ie1[dd - 1] = top; }
    SETR(1, R->ieu + 1)
    for (int k = is1[2]; k <= ie1[2]; k++) for (int j = is1[1]; j <= ie1[1]; j++) for (int i = is1[0]; i <= ie1[0]; i++) {
        if (u[IX(i - i0, j, k)] + u[IX(i, j + j0, k + k0)] > 0.0)
            W1[IX(i, j, k)] = phi[IX(i - i0, j, k)] +
                0.5 * slope_lim(phi[IX(i - 1 - i0, j, k)], phi[IX(i - i0, j, k)], phi[IX(i + 1 - i0, j, k)], scheme);
        else
            W1[IX(i, j, k)] = phi[IX(i + 1 - i0, j, k)] -
                0.5 * slope_lim(phi[IX(i - i0, j, k)], phi[IX(i + 1 - i0, j, k)], phi[IX(i + 2 - i0, j, k)], scheme);
    }
    SETR(2, R->jev + 1)
    for (int k = is1[2]; k <= ie1[2]; k++) for (int j = is1[1]; j <= ie1[1]; j++) for (int i = is1[0]; i <= ie1[0]; i++) {
        if (v[IX(i, j - j0, k)] + v[IX(i + i0, j, k + k0)] > 0.0)
            W2[IX(i, j, k)] = phi[IX(i, j - j0, k)] +
                0.5 * slope_lim(phi[IX(i, j - 1 - j0, k)], phi[IX(i, j - j0, k)], phi[IX(i, j + 1 - j0, k)], scheme);
        else
            W2[IX(i, j, k)] = phi[IX(i, j + 1 - j0, k)] -
                0.5 * slope_lim(phi[IX(i, j - j0, k)], phi[IX(i, j + 1 - j0, k)], phi[IX(i, j + 2 - j0, k)], scheme);
    }
    SETR(3, R->kew + 1)
    for (int k = is1[2]; k <= ie1[2]; k++) for (int j = is1[1]; j <= ie1[1]; j++) for (int i = is1[0]; i <= ie1[0]; i++) {
        if (w[IX(i, j, k - k0)] + w[IX(i + i0, j + j0, k)] > 0.0)
            W3[IX(i, j, k)] = phi[IX(i, j, k - k0)] +
                0.5 * slope_lim(phi[IX(i, j, k - 1 - k0)], phi[IX(i, j, k - k0)], phi[IX(i, j, k + 1 - k0)], scheme);
        else
            W3[IX(i, j, k)] = phi[IX(i, j, k + 1 - k0)] -
                0.5 * slope_lim(phi[IX(i, j, k - k0)], phi[IX(i, j, k + 1 - k0)], phi[IX(i, j, k + 2 - k0)], scheme);
    }
#undef SETR
    for (int q = 0; q < 3; q++) { is1[q] = is0[q] + 1; ie1[q] = ie0[q]; }
    if (d == 1) ie1[0] = R->ieu;
    else if (d == 2) ie1[1] = R->jev;
    else ie1[2] = R->kew;
    for (int k = is1[2]; k <= ie1[2]; k++) for (int j = is1[1]; j <= ie1[1]; j++) for (int i = is1[0]; i <= ie1[0]; i++) {
        dphi[IX(i, j, k)] =
            -0.5 * ((u[IX(i, j, k)] + u[IX(i + i0, j + j0, k + k0)]) * W1[IX(i + i0, j, k)] -
                    (u[IX(i - 1 + i0, j, k)] + u[IX(i - 1, j + j0, k + k0)]) * W1[IX(i - 1 + i0, j, k)]) / dx[i]
            - 0.5 * ((v[IX(i, j, k)] + v[IX(i + i0, j + j0, k + k0)]) * W2[IX(i, j + j0, k)] -
                     (v[IX(i, j - 1 + j0, k)] + v[IX(i + i0, j - 1, k + k0)]) * W2[IX(i, j - 1 + j0, k)]) / dy[j]
            - 0.5 * ((w[IX(i, j, k)] + w[IX(i + i0, j + j0, k + k0)]) * W3[IX(i, j, k + k0)] -
                     (w[IX(i, j, k - 1 + k0)] + w[IX(i + i0, j + j0, k - 1)]) * W3[IX(i, j, k - 1 + k0)]) / dz[k];
    }
}

/* momentumConvection (paris.f90:1957-1984): scheme 0 QUICK, 1 ENO,
 * 2 Superbee, 3 WENO */
int og_momentum_convection(const paris_grid_desc* desc, int scheme, const double* u, const double* v,
                           const double* w, double* du, double* dv, double* dw) {
    if (scheme == 0) return og_momentum_convection_quick(desc, u, v, w, du, dv, dw);
    if (scheme < 1 || scheme > 3) return PARIS_BAD_ARGS;
    og_grid* g = og_grid_new(desc);
    mom_rng R;
    rng_init(&R, g);
    double* W1 = calloc(g->ntot, sizeof(double));
    double* W2 = calloc(g->ntot, sizeof(double));
    double* W3 = calloc(g->ntot, sizeof(double));
    conv_onedim(g, &R, u, v, w, u, du, 1, scheme, W1, W2, W3);
    conv_onedim(g, &R, u, v, w, v, dv, 2, scheme, W1, W2, W3);
    conv_onedim(g, &R, u, v, w, w, dw, 3, scheme, W1, W2, W3);
    free(W1); free(W2); free(W3);
    og_grid_free(g);
    return 0;
}

/* explicitMomDiff, paris.f90:2757-2808 (adds to du, dv, dw) */
int og_explicit_mom_diff(const paris_grid_desc* desc, const double* u, const double* v, const double* w,
                         const double* rho, const double* mu, double* du, double* dv, double* dw) {
    og_grid* g = og_grid_new(desc);
    mom_rng R;
    rng_init(&R, g);
    const double *dx = g->dx, *dxh = g->dxh, *dy = g->dy, *dyh = g->dyh, *dz = g->dz, *dzh = g->dzh;
#define U(i, j, k) u[IX(i, j, k)]
#define V(i, j, k) v[IX(i, j, k)]
#define W(i, j, k) w[IX(i, j, k)]
#define M(i, j, k) mu[IX(i, j, k)]
#define RH(i, j, k) rho[IX(i, j, k)]
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ieu; i++) {
        du[IX(i, j, k)] = du[IX(i, j, k)] + (
            (1. / dxh[i]) * 2. * (M(i + 1, j, k) * (1. / dx[i + 1]) * (U(i + 1, j, k) - U(i, j, k)) -
                                  M(i, j, k) * (1. / dx[i]) * (U(i, j, k) - U(i - 1, j, k)))
            + (1. / dy[j]) * (0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j + 1, k) + M(i, j + 1, k)) *
                                  ((1. / dyh[j]) * (U(i, j + 1, k) - U(i, j, k)) + (1. / dxh[i]) * (V(i + 1, j, k) - V(i, j, k))) -
                              0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j - 1, k) + M(i, j - 1, k)) *
                                  ((1. / dyh[j - 1]) * (U(i, j, k) - U(i, j - 1, k)) + (1. / dxh[i]) * (V(i + 1, j - 1, k) - V(i, j - 1, k))))
            + (1. / dz[k]) * (0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j, k + 1) + M(i, j, k + 1)) *
                                  ((1. / dzh[k]) * (U(i, j, k + 1) - U(i, j, k)) + (1. / dxh[i]) * (W(i + 1, j, k) - W(i, j, k))) -
                              0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j, k - 1) + M(i, j, k - 1)) *
                                  ((1. / dzh[k - 1]) * (U(i, j, k) - U(i, j, k - 1)) + (1. / dxh[i]) * (W(i + 1, j, k - 1) - W(i, j, k - 1))))
            ) / (0.5 * (RH(i + 1, j, k) + RH(i, j, k)));
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.jev; j++) for (int i = R.is; i <= R.ie; i++) {
        dv[IX(i, j, k)] = dv[IX(i, j, k)] + (
            (1. / dx[i]) * (0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j + 1, k) + M(i, j + 1, k)) *
                                ((1. / dyh[j]) * (U(i, j + 1, k) - U(i, j, k)) + (1. / dxh[i]) * (V(i + 1, j, k) - V(i, j, k))) -
                            0.25 * (M(i, j, k) + M(i, j + 1, k) + M(i - 1, j + 1, k) + M(i - 1, j, k)) *
                                ((1. / dyh[j]) * (U(i - 1, j + 1, k) - U(i - 1, j, k)) + (1. / dxh[i - 1]) * (V(i, j, k) - V(i - 1, j, k))))
            + (1. / dyh[j]) * 2. * (M(i, j + 1, k) * (1. / dy[j + 1]) * (V(i, j + 1, k) - V(i, j, k)) -
                                    M(i, j, k) * (1. / dy[j]) * (V(i, j, k) - V(i, j - 1, k)))
            + (1. / dz[k]) * (0.25 * (M(i, j, k) + M(i, j + 1, k) + M(i, j + 1, k + 1) + M(i, j, k + 1)) *
                                  ((1. / dzh[k]) * (V(i, j, k + 1) - V(i, j, k)) + (1. / dyh[j]) * (W(i, j + 1, k) - W(i, j, k))) -
                              0.25 * (M(i, j, k) + M(i, j + 1, k) + M(i, j + 1, k - 1) + M(i, j, k - 1)) *
                                  ((1. / dzh[k - 1]) * (V(i, j, k) - V(i, j, k - 1)) + (1. / dyh[j]) * (W(i, j + 1, k - 1) - W(i, j, k - 1))))
            ) / (0.5 * (RH(i, j + 1, k) + RH(i, j, k)));
    }
    for (int k = R.ks; k <= R.kew; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        dw[IX(i, j, k)] = dw[IX(i, j, k)] + (
            (1. / dx[i]) * (0.25 * (M(i, j, k) + M(i + 1, j, k) + M(i + 1, j, k + 1) + M(i, j, k + 1)) *
                                ((1. / dzh[k]) * (U(i, j, k + 1) - U(i, j, k)) + (1. / dxh[i]) * (W(i + 1, j, k) - W(i, j, k))) -
                            0.25 * (M(i, j, k) + M(i - 1, j, k) + M(i - 1, j, k + 1) + M(i, j, k + 1)) *
                                ((1. / dzh[k]) * (U(i - 1, j, k + 1) - U(i - 1, j, k)) + (1. / dxh[i - 1]) * (W(i, j, k) - W(i - 1, j, k))))
            + (1. / dy[j]) * (0.25 * (M(i, j, k) + M(i, j + 1, k) + M(i, j + 1, k + 1) + M(i, j, k + 1)) *
                                  ((1. / dzh[k]) * (V(i, j, k + 1) - V(i, j, k)) + (1. / dyh[j]) * (W(i, j + 1, k) - W(i, j, k))) -
                              0.25 * (M(i, j, k) + M(i, j - 1, k) + M(i, j - 1, k + 1) + M(i, j, k + 1)) *
                                  ((1. / dzh[k]) * (V(i, j - 1, k + 1) - V(i, j - 1, k)) + (1. / dyh[j - 1]) * (W(i, j, k) - W(i, j - 1, k))))
            + (1. / dzh[k]) * 2. * (M(i, j, k + 1) * (1. / dz[k + 1]) * (W(i, j, k + 1) - W(i, j, k)) -
                                    M(i, j, k) * (1. / dz[k]) * (W(i, j, k) - W(i, j, k - 1)))
            ) / (0.5 * (RH(i, j, k + 1) + RH(i, j, k)));
    }
#undef U
#undef V
#undef W
#undef M
#undef RH
    og_grid_free(g);
    return 0;
}

/* volumeForce, paris.f90:2813-2860, with the front-tracking force fx, fy,
 * fz zero as the step loop leaves them (paris.f90:396-398) */
int og_volume_force(const paris_grid_desc* desc, const double* rho, double dpdx, double dpdy, double dpdz,
                    int buoyancy, double gx, double gy, double gz, double rho_ave, double* du, double* dv,
                    double* dw) {
    double rro;
    if (buoyancy == 0) rro = 0.0;
    else if (buoyancy == 1) rro = desc->rho1;
    else if (buoyancy == 2) rro = desc->rho2;
    else if (buoyancy == 3) rro = rho_ave;
    else return PARIS_BAD_ARGS;
    og_grid* g = og_grid_new(desc);
    mom_rng R;
    rng_init(&R, g);
    const long sx = 1, sy = g->sy, sz = g->sz;
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ieu; i++) {
        long n = IX(i, j, k);
        double fx = 0.0 - dpdx + (0.5 * (rho[n + sx] + rho[n]) - rro) * gx;
        du[n] = du[n] + fx / (0.5 * (rho[n + sx] + rho[n]));
    }
    for (int k = R.ks; k <= R.ke; k++) for (int j = R.js; j <= R.jev; j++) for (int i = R.is; i <= R.ie; i++) {
        long n = IX(i, j, k);
        double fy = 0.0 - dpdy + (0.5 * (rho[n + sy] + rho[n]) - rro) * gy;
        dv[n] = dv[n] + fy / (0.5 * (rho[n + sy] + rho[n]));
    }
    for (int k = R.ks; k <= R.kew; k++) for (int j = R.js; j <= R.je; j++) for (int i = R.is; i <= R.ie; i++) {
        long n = IX(i, j, k);
        double fz = 0.0 - dpdz + (0.5 * (rho[n + sz] + rho[n]) - rro) * gz;
        dw[n] = dw[n] + fz / (0.5 * (rho[n + sz] + rho[n]));
    }
    og_grid_free(g);
    return 0;
}

/* u = u + dt*du over whole arrays, paris.f90:442-444 */
int og_advance_velocity(const paris_grid_desc* desc, double dt, double* u, double* v, double* w, const double* du,
                        const double* dv, const double* dw) {
    og_grid* g = og_grid_new(desc);
    for (long n = 0; n < g->ntot; n++) {
        u[n] = u[n] + dt * du[n];
        v[n] = v[n] + dt * dv[n];
        w[n] = w[n] + dt * dw[n];
    }
    og_grid_free(g);
    return 0;
}

/* SetVelocityBC (modules.f90:951-973, 1061-1105) for periodic and no-slip /
 * moving-wall boundaries, then do_ghost_vector (modules.f90:1628-1642).
 * wallvel: WallVel(6,3) in Fortran order (face f, component c at
 * (f-1) + 6*(c-1)), NULL for zero. */
int og_set_velocity_bc(const paris_grid_desc* desc, double* u, double* v, double* w, const double* wallvel) {
    for (int f = 0; f < 6; f++)
        if (desc->bdry_cond[f] != PARIS_BC_WALL && desc->bdry_cond[f] != PARIS_BC_PERIODIC) return PARIS_BAD_ARGS;
    og_grid* g = og_grid_new(desc);
    mom_rng R;
    rng_init(&R, g);
    double WV[18] = {0};
    if (wallvel) memcpy(WV, wallvel, sizeof(WV));
#define WVEL(f, c) WV[((f) - 1) + 6 * ((c) - 1)]
    const int nxt = g->Nt[0], nyt = g->Nt[1], nzt = g->Nt[2];
    const int is = R.is, ie = R.ie, js = R.js, je = R.je, ks = R.ks, ke = R.ke;
    if (desc->bdry_cond[0] == PARIS_BC_WALL)
        for (int k = 0; k < nzt; k++) for (int j = 0; j < nyt; j++) {
            u[IX(is - 1, j, k)] = 0.0;
            u[IX(is - 2, j, k)] = -u[IX(is, j, k)];
            v[IX(is - 1, j, k)] = 2 * WVEL(1, 2) - v[IX(is, j, k)];
            w[IX(is - 1, j, k)] = 2 * WVEL(1, 3) - w[IX(is, j, k)];
        }
    if (desc->bdry_cond[3] == PARIS_BC_WALL)
        for (int k = 0; k < nzt; k++) for (int j = 0; j < nyt; j++) {
            u[IX(ie, j, k)] = 0.0;
            u[IX(ie + 1, j, k)] = -u[IX(ie - 1, j, k)];
            v[IX(ie + 1, j, k)] = 2 * WVEL(2, 2) - v[IX(ie, j, k)];
            w[IX(ie + 1, j, k)] = 2 * WVEL(2, 3) - w[IX(ie, j, k)];
        }
    if (desc->bdry_cond[1] == PARIS_BC_WALL)
        for (int k = 0; k < nzt; k++) for (int i = 0; i < nxt; i++) {
            v[IX(i, js - 1, k)] = 0.0;
            v[IX(i, js - 2, k)] = -v[IX(i, js, k)];
            u[IX(i, js - 1, k)] = 2 * WVEL(3, 1) - u[IX(i, js, k)];
            w[IX(i, js - 1, k)] = 2 * WVEL(3, 3) - w[IX(i, js, k)];
        }
    if (desc->bdry_cond[4] == PARIS_BC_WALL)
        for (int k = 0; k < nzt; k++) for (int i = 0; i < nxt; i++) {
            v[IX(i, je, k)] = 0.0;
            v[IX(i, je + 1, k)] = -v[IX(i, je - 1, k)];
            u[IX(i, je + 1, k)] = 2 * WVEL(4, 1) - u[IX(i, je, k)];
            w[IX(i, je + 1, k)] = 2 * WVEL(4, 3) - w[IX(i, je, k)];
        }
    if (desc->bdry_cond[2] == PARIS_BC_WALL)
        for (int j = 0; j < nyt; j++) for (int i = 0; i < nxt; i++) {
            w[IX(i, j, ks - 1)] = 0.0;
            w[IX(i, j, ks - 2)] = -w[IX(i, j, ks)];
            u[IX(i, j, ks - 1)] = 2 * WVEL(5, 1) - u[IX(i, j, ks)];
            v[IX(i, j, ks - 1)] = 2 * WVEL(5, 2) - v[IX(i, j, ks)];
        }
    if (desc->bdry_cond[5] == PARIS_BC_WALL)
        for (int j = 0; j < nyt; j++) for (int i = 0; i < nxt; i++) {
            w[IX(i, j, ke)] = 0.0;
            w[IX(i, j, ke + 1)] = -w[IX(i, j, ke - 1)];
            u[IX(i, j, ke + 1)] = 2 * WVEL(6, 1) - u[IX(i, j, ke)];
            v[IX(i, j, ke + 1)] = 2 * WVEL(6, 2) - v[IX(i, j, ke)];
        }
#undef WVEL
    og_do_all_ghost(g, u);
    og_do_all_ghost(g, v);
    og_do_all_ghost(g, w);
    og_grid_free(g);
    return 0;
}
