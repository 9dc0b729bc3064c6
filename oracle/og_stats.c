/*
 * og_stats.c -- oracle of the time-step control and the flow statistics
 * (test infrastructure only): TimeStepSize without a free surface
 * (paris.f90:968-1041), get_cfl_and_check (paris.f90:1045-1074) and calcStats
 * (paris.f90:1116-1267), in the reference's loop order (k, j, i).
 *
 * Arrays are ghosted, C index = Fortran index - 1 (interior [ng, ng+n)).
 * Expressions keep the Fortran operation order (x**2 is x*x; the Fortran
 * single-precision literals 0.5 and 2.0 are exact).  uold is zero, as the
 * reference keeps it only for itime_scheme 2 (paris.f90:267-273).
 */
#include <math.h>
#include <string.h>

#include "og.h"

#define IX(i, j, k) OG_IX(g, i, j, k)

/* vmax = maxval(sqrt(u**2+v**2+w**2)) over the interior (paris.f90:1016) */
static double vmax_interior(const og_grid* g, const double* u, const double* v, const double* w) {
    double vmax = 0.0;
    for (int k = g->ng; k < g->ng + g->nz; k++)
        for (int j = g->ng; j < g->ng + g->ny; j++)
            for (int i = g->ng; i < g->ng + g->nx; i++) {
                long n = IX(i, j, k);
                double vl = sqrt(u[n] * u[n] + v[n] * v[n] + w[n] * w[n]);
                if (vl > vmax) vmax = vl;
            }
    return vmax;
}

/* h = minval(dx) over dx(imin:imax) */
static double min_dx(const og_grid* g) {
    double h = g->dx[0];
    for (int i = 1; i < g->Nt[0]; i++) h = og_dmin1(h, g->dx[i]);
    return h;
}

/* TimeStepSize(deltaT, vof_phase), paris.f90:968-1041, FreeSurface false */
int og_time_step_size(const paris_grid_desc* desc, const double* u, const double* v, const double* w, double cfl,
                      double max_dt, double u_inject, double* dt, double* vmax_out) {
    og_grid* g = og_grid_new(desc);
    if (!g) return PARIS_BAD_ARGS;
    double vmax_phys = og_dmax1(1e-3, u_inject);
    double h = min_dx(g);
    double vmax = vmax_interior(g, u, v, w);
    double dtadv = h / og_dmax1(vmax_phys, vmax);
    double mydt = cfl * dtadv;
    mydt = og_dmin1(mydt, max_dt);
    *dt = mydt;
    if (vmax_out) *vmax_out = vmax;
    og_grid_free(g);
    return PARIS_OK;
}

/* get_cfl_and_check(deltaT), paris.f90:1045-1074 */
int og_get_cfl_and_check(const paris_grid_desc* desc, const double* u, const double* v, const double* w, double dt,
                         double cflmax_allowed, double* cfl) {
    og_grid* g = og_grid_new(desc);
    if (!g) return PARIS_BAD_ARGS;
    double vmax = vmax_interior(g, u, v, w);
    double h = min_dx(g);
    *cfl = vmax * dt / h;
    og_grid_free(g);
    return *cfl > cflmax_allowed ? PARIS_CFL_TOO_LARGE : PARIS_OK;
}

/* accumulate a term into column q (1-based) and its absolute value */
#define ADD(q, val)                         \
    do {                                    \
        double _t = (val);                  \
        ms[(q)-1] = ms[(q)-1] + _t;         \
        if (ab) ab[(q)-1] += fabs(_t);      \
    } while (0)

/* calcStats, paris.f90:1116-1267, DoVOF true.  abs_out (may be NULL)
 * receives the sums of |term| per column before the normalisations, the
 * scale of the rounding error of a reordered sum. */
int og_calc_stats(const paris_grid_desc* desc, const double* u, const double* v, const double* w,
                  const double* rho, const double* p, const double* cvof, const double* mu,
                  const int32_t* flag, const paris_stats_opts* o, double* stats, double* abs_out) {
    og_grid* g = og_grid_new(desc);
    if (!g) return PARIS_BAD_ARGS;
    paris_stats_opts z;
    memset(&z, 0, sizeof z);
    if (!o) o = &z;
    const int tb = o->test_flags & PARIS_STATS_RISING_BUBBLE, tpi = o->test_flags & PARIS_STATS_PHASE_INVERSION,
              tt = o->test_flags & PARIS_STATS_TURB;
    double rro = 0.0;
    if (o->buoyancy_case == 1) rro = desc->rho1;
    else if (o->buoyancy_case == 2) rro = desc->rho2;
    else if (o->buoyancy_case == 3) rro = o->rho_ave;
    else if (o->buoyancy_case != 0) { og_grid_free(g); return PARIS_BAD_ARGS; }
    const int is = g->ng, ie = g->ng + g->nx - 1, js = g->ng, je = g->ng + g->ny - 1, ks = g->ng,
              ke = g->ng + g->nz - 1;
    const int ieu = ie - (og_is_periodic(g, 0) ? 0 : 1), jev = je - (og_is_periodic(g, 1) ? 0 : 1),
              kew = ke - (og_is_periodic(g, 2) ? 0 : 1);
    const double xl = desc->xlength, yl = desc->ylength, zl = desc->zlength;
    const double height4stats = 0.875;
    double ms[PARIS_NSTATS], abv[PARIS_NSTATS];
    double* ab = abs_out ? abv : NULL;
    memset(ms, 0, sizeof ms);
    memset(abv, 0, sizeof abv);
    const double *x = g->x, *y = g->y, *z_ = g->z;
    for (int k = ks; k <= ke; k++)
        for (int j = js; j <= je; j++)
            for (int i = is; i <= ie; i++) {
                long n = IX(i, j, k);
                long e = 1, nn = g->sy, t = g->sz;
                double vol = g->dx[i] * g->dy[j] * g->dz[k];
                ADD(2, u[n] * vol);
                /* fx, fy, fz as volumeForce left them (paris.f90:395-397, 2841-2857) */
                double fx = 0.0, fy = 0.0, fz = 0.0;
                if (o->force_valid) {
                    if (i <= ieu) fx = 0.0 - o->dpdx + (0.5 * (rho[n + e] + rho[n]) - rro) * o->gx;
                    if (j <= jev) fy = 0.0 - o->dpdy + (0.5 * (rho[n + nn] + rho[n]) - rro) * o->gy;
                    if (k <= kew) fz = 0.0 - o->dpdz + (0.5 * (rho[n + t] + rho[n]) - rro) * o->gz;
                }
                ADD(3, fx * g->dxh[i] * g->dy[j] * g->dz[k]);
                ADD(4, fy * g->dx[i] * g->dyh[j] * g->dz[k]);
                ADD(5, fz * g->dx[i] * g->dy[j] * g->dzh[k]);
                ADD(6, rho[n] * vol);
                ADD(7, p[n] * vol);
                ADD(8, 0.5 * (rho[n] + rho[n + e]) * u[n] * vol);
                ADD(9, 0.5 * (rho[n] + rho[n + e]) * 0.0 * vol);
                double cc = cvof[n];
                ADD(10, cc * vol);
                ADD(11, cc * vol * x[i]);
                if (tb) ADD(24, 0.50 * (u[n - e] + u[n]) * cc * vol);
                double a1 = 0.5 * (u[n] + u[n + e]), a2 = 0.5 * (v[n] + v[n + nn]), a3 = 0.5 * (w[n] + w[n + t]);
                double kenergy = 0.5 * (a1 * a1 + a2 * a2 + a3 * a3);
                ADD(12, rho[n] * kenergy * vol * cvof[n]);
                ADD(13, rho[n] * kenergy * vol * (1.0 - cvof[n]));
                if (tt) {
                    double b1 = (-u[n] + u[n + e]) / g->dx[i], b2 = (-v[n] + v[n + nn]) / g->dy[j];
                    ADD(14, b1 * b1 * vol);
                    ADD(15, b2 * b2 * vol);
                } else {
                    ADD(14, rho[n] * 0.5 * (v[n] + v[n + nn]) * vol * (cvof[n]));
                    ADD(15, rho[n] * 0.5 * (v[n] + v[n + nn]) * vol * (1.0 - cvof[n]));
                }
                if (cc > 0.0 && cc < 1.0) {
                    double st[27], m[3];
                    for (int c = -1; c <= 1; c++)
                        for (int b = -1; b <= 1; b++)
                            for (int a = -1; a <= 1; a++) st[OG_C3(a + 1, b + 1, c + 1)] = cvof[IX(i + a, j + b, k + c)];
                    og_mycs(st, m);
                    if (m[0] != 0.0 || m[1] != 0.0 || m[2] != 0.0) ADD(19, og_area3d(m, cc));
                }
                if (tpi) {
                    ADD(20, rho[n] * o->gy * y[j] * vol * cvof[n]);
                    ADD(21, rho[n] * o->gy * y[j] * vol * (1.0 - cvof[n]));
                }
                double d1 = 0.5 * (w[n + nn] + w[n + nn + t] - w[n - nn] - w[n - nn + t]) / (y[j + 1] - y[j - 1]) -
                            0.5 * (v[n + t] + v[n + nn + t] - v[n - t] - v[n + nn - t]) / (z_[k + 1] - z_[k - 1]);
                double d2 = 0.5 * (u[n + t] + u[n + e + t] - u[n - t] - u[n + e - t]) / (z_[k + 1] - z_[k - 1]) -
                            0.5 * (w[n + e] + w[n + e + t] - w[n - e] - w[n - e + t]) / (x[i + 1] - x[i - 1]);
                double d3 = 0.5 * (v[n + e] + v[n + e + nn] - v[n - e] - v[n - e + nn]) / (x[i + 1] - x[i - 1]) -
                            0.5 * (u[n + nn] + u[n + e + nn] - u[n - nn] - u[n + e - nn]) / (y[j + 1] - y[j - 1]);
                double vort2 = d1 * d1 + d2 * d2 + d3 * d3;
                double enstrophy = 0.5 * vort2;
                ADD(22, enstrophy * vol * cvof[n]);
                ADD(23, enstrophy * vol * (1.0 - cvof[n]));
                if (flag[n] == 2) ADD(25, 1.0);
                if (tpi && y[j] > height4stats) ADD(24, vol * cvof[n] / (xl * zl * (yl - height4stats)));
            }
    /* shear stress on y = 0 and y = Ly (js == Ng+1, je == Ng+Ny on one rank) */
    for (int k = ks; k <= ke; k++)
        for (int i = is; i <= ie; i++) {
            long n = IX(i, js, k);
            ADD(1, mu[n] * u[n] * g->dx[i] * g->dz[k] / (g->dy[js] / 2.0));
        }
    for (int k = ks; k <= ke; k++)
        for (int i = is; i <= ie; i++) {
            long n = IX(i, je, k);
            ADD(1, mu[n] * u[n] * g->dx[i] * g->dz[k] / (g->dy[je] / 2.0));
        }
    /* pressure at entry and exit: p(ng+1, ny/2+ng, nz/2+ng), p(ng+nx, ...) */
    int jp = g->ny / 2 + g->ng - 1, kp = g->nz / 2 + g->ng - 1;
    ms[16] = p[IX(is, jp, kp)];
    ms[17] = p[IX(ie, jp, kp)];
    double V = xl * yl * zl;
    for (int q = 1; q < 11; q++) ms[q] = ms[q] / V;
    ms[0] = ms[0] / (xl * zl * 2.0);
    if (tb) {
        ms[9] = ms[9] * V;
        ms[10] = ms[10] * V;
        if (ms[9] > 1e-15) {
            ms[10] = ms[10] / ms[9];
            ms[23] = ms[23] / ms[9];
        }
    }
    memcpy(stats, ms, sizeof ms);
    if (abs_out) memcpy(abs_out, abv, sizeof abv);
    og_grid_free(g);
    return PARIS_OK;
}
