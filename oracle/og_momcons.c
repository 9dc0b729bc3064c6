/*
 * og_momcons.c -- oracle (test infrastructure only) of the momentum-conserving
 * VOF sweeps of DoMOMCONS: vofandmomsweepsstaggered (vofmodules.f90:1536-1692)
 * with, per momentum component dir,
 *   staggered (staggeredmom = T):
 *     get_momentum_staggered (vofmodules.f90:1396-1449, get_half_fractions
 *     :1307-1338), then for the three split directions d in the order of
 *     MOD(tswap,3): swpmom_stg (vofnonmodule.f90:96-116: swpzmom_stg
 *     :433-631 or swprmom_stg :966-1139) and swp_stg (:50-71: swpz_stg
 *     :239-331 or swpr_stg :757-855), then get_velocity_from_momentum_staggered
 *     (vofmodules.f90:1486-1534);
 *   centred (staggeredmom = F):
 *     get_momentum_centered (:1363-1394), swpmom (vofnonmodule.f90:74-94:
 *     swpzmom :333-431 or swprmom :856-962) and swp, then
 *     get_velocity_from_momentum_centered (vofmodules.f90:1451-1484),
 * and SetMomentumBC (modules.f90:1329-1625) for periodic and wall boundaries.
 * Loops keep the reference's ranges ([is-1, ie+1] boxes) and operation order.
 *
 * The swp_stg sweeps are swpz / swpr with the face velocity
 * 0.5*(us(i) + us(i+e_dir)) in place of us(i): that average is formed into an
 * array first (the same two operations), then the plain sweep runs on it.
 *
 * Two points where the reference reads values it never set are made
 * definite here and on the device alike:
 *   - the `momentum` array is zero when first allocated, and keeps its ghost
 *     values between calls (cells no loop or boundary condition writes);
 *   - with LinInterp, a cell whose complementary plane fit fails (zero
 *     normal of 1 - c) takes the complement of its own plane, -nr and
 *     -alpha (the reference keeps nrc and alphac of an earlier cell).
 * The solid mask of SetMomentumBC is 1 everywhere (no obstacles), so
 * u = u*mask and mom = mom*mask change nothing and are left out.
 *
 * One deliberate change: the staggered fraction 0.5*(work2(i) +
 * work1(i+e_dir)) is clipped to [0, 1].  A half fraction of a nearly full
 * cell can round to just above 1, and a fraction above 1 sends AL3D into the
 * cube root of a negative number (NaN) in the first sweep; whether that
 * happens depends on the last bit of the plane constant, so without the clip
 * two correct implementations of AL3D disagree between a number and NaN.
 */
#include <math.h>
#include <string.h>

#include "og.h"

typedef struct {
    og_grid* g;
    double dt, dxyz, rho1, rho2;
    int scheme, lin;
    double wv[18];   /* WallVel(6,3), face f component c at (f-1)+6*(c-1) */
} mc_ctx;

#define WV(m, f, c) ((m)->wv[((f) - 1) + 6 * ((c) - 1)])

static double minabs(double a, double b) { return fabs(a) < fabs(b) ? a : b; }
static double maxabs(double a, double b) { return fabs(a) > fabs(b) ? a : b; }

/* slope_lim (modules.f90:177-197) and interpole3 (:199-206) */
static double interpole3(double v1, double v2, double v3, int scheme, double delta_x) {
    double s = 0.0;
    if (scheme == PARIS_CONV_SUPERBEE) {
        double a1 = minabs(v3 - v2, 2.0 * (v2 - v1));
        double a2 = minabs(2.0 * (v3 - v2), v2 - v1);
        s = maxabs(a1, a2);
    } else if (scheme == PARIS_CONV_ENO) {
        s = minabs(v3 - v2, v2 - v1);
    } else if (scheme == PARIS_CONV_WENO) {
        double d1 = v2 - v1, d2 = v3 - v2;
        double a1 = 1.0 / (d1 * d1 + 1.e-16);
        double a2 = 1.0 / (d2 * d2 + 1.e-16);
        double a = a1 + a2;
        s = (a1 * (v2 - v1) + a2 * (v3 - v2)) / a;
    }
    return v2 + s * delta_x;
}

static double rho_of(const mc_ctx* m, double c) { return m->rho2 * c + m->rho1 * (1.0 - c); }

/* SetMomentumBC(u, c, mom, d, mask, rho1, rho2, t), modules.f90:1329-1625,
 * for walls (bdry_cond 0) on one rank; d is 0..2.  The x+ tangential line
 * raises to a power, as the reference writes it. */
static void set_momentum_bc(const mc_ctx* m, const double* u, const double* c, double* mom, int d) {
    const og_grid* g = m->g;
    const int ng = g->ng;
    const int is = ng, ie = ng + g->nx - 1, js = ng, je = ng + g->ny - 1, ks = ng, ke = ng + g->nz - 1;
    const int NI = g->Nt[0], NJ = g->Nt[1], NK = g->Nt[2];
#define IXg(i, j, k) OG_IX(g, i, j, k)
    if (g->d.bdry_cond[0] == PARIS_BC_WALL)
        for (int k = 0; k < NK; k++)
            for (int j = 0; j < NJ; j++) {
                if (d == 0) {
                    mom[IXg(is - 1, j, k)] = 0.0;
                    mom[IXg(is - 2, j, k)] = -mom[IXg(is, j, k)];
                } else {
                    mom[IXg(is - 1, j, k)] = (2 * WV(m, 1, 2) - u[IXg(is, j, k)]) * rho_of(m, c[IXg(is, j, k)]);
                }
            }
    if (g->d.bdry_cond[3] == PARIS_BC_WALL)
        for (int k = 0; k < NK; k++)
            for (int j = 0; j < NJ; j++) {
                if (d == 0) {
                    mom[IXg(ie, j, k)] = 0.0;
                    mom[IXg(ie + 1, j, k)] = -mom[IXg(ie - 1, j, k)];
                } else {
                    mom[IXg(ie + 1, j, k)] = pow(2 * WV(m, 2, 2) - u[IXg(ie, j, k)], rho_of(m, c[IXg(ie, j, k)]));
                }
            }
    if (g->d.bdry_cond[1] == PARIS_BC_WALL)
        for (int k = 0; k < NK; k++)
            for (int i = 0; i < NI; i++) {
                if (d == 1) {
                    mom[IXg(i, js - 1, k)] = 0.0;
                    mom[IXg(i, js - 2, k)] = -mom[IXg(i, js, k)];
                } else {
                    mom[IXg(i, js - 1, k)] = (2 * WV(m, 3, 1) - u[IXg(i, js, k)]) * rho_of(m, c[IXg(i, js, k)]);
                }
            }
    if (g->d.bdry_cond[4] == PARIS_BC_WALL)
        for (int k = 0; k < NK; k++)
            for (int i = 0; i < NI; i++) {
                if (d == 1) {
                    mom[IXg(i, je, k)] = 0.0;
                    mom[IXg(i, je + 1, k)] = -mom[IXg(i, je - 1, k)];
                } else {
                    mom[IXg(i, je + 1, k)] = (2 * WV(m, 4, 1) - u[IXg(i, je, k)]) * rho_of(m, c[IXg(i, je, k)]);
                }
            }
    if (g->d.bdry_cond[2] == PARIS_BC_WALL)
        for (int j = 0; j < NJ; j++)
            for (int i = 0; i < NI; i++) {
                if (d == 2) {
                    mom[IXg(i, j, ks - 1)] = 0.0;
                    mom[IXg(i, j, ks - 2)] = -mom[IXg(i, j, ks)];
                } else {
                    mom[IXg(i, j, ks - 1)] = (2 * WV(m, 5, 1) - u[IXg(i, j, ks)]) * rho_of(m, c[IXg(i, j, ks)]);
                }
            }
    if (g->d.bdry_cond[5] == PARIS_BC_WALL)
        for (int j = 0; j < NJ; j++)
            for (int i = 0; i < NI; i++) {
                if (d == 2) {
                    mom[IXg(i, j, ke)] = 0.0;
                    mom[IXg(i, j, ke + 1)] = -mom[IXg(i, j, ke - 1)];
                } else {
                    mom[IXg(i, j, ke + 1)] = (2 * WV(m, 6, 1) - u[IXg(i, j, ke)]) * rho_of(m, c[IXg(i, j, ke)]);
                }
            }
#undef IXg
}

/* the [is-1, ie+1]^3 box of the reference's flux loops */
#define BOX_LOOP(g)                                              \
    for (int k = (g)->ng - 1; k <= (g)->ng + (g)->nz; k++)       \
        for (int j = (g)->ng - 1; j <= (g)->ng + (g)->ny; j++)   \
            for (int i = (g)->ng - 1; i <= (g)->ng + (g)->nx; i++)
#define INT_LOOP(g)                                              \
    for (int k = (g)->ng; k < (g)->ng + (g)->nz; k++)            \
        for (int j = (g)->ng; j < (g)->ng + (g)->ny; j++)        \
            for (int i = (g)->ng; i < (g)->ng + (g)->nx; i++)

/* get_half_fractions(c, d, i, j, k, vofh1, vofh2), vofmodules.f90:1307-1338 */
static void half_fractions(const og_grid* g, const double* c, long n, int d, double* h1, double* h2) {
    *h1 = c[n];
    *h2 = c[n];
    if (c[n] > 0.0 && c[n] < 1.0) {
        double st[27], dm[3], alpha, x0[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0};
        og_stencil(g, c, n, st);
        if (og_fit_plane_new(c[n], d, 0.0, 0.0, st, dm, &alpha)) return;
        dx[d] = 0.5;
        *h1 = 2.0 * og_fl3d(dm, alpha, x0, dx);
        x0[d] = 0.5;
        *h2 = 2.0 * og_fl3d(dm, alpha, x0, dx);
    }
}

/* swpzmom_stg (staggered = 1, vofnonmodule.f90:433-631) or swpzmom
 * (staggered = 0, :333-431): the CIAM fluxes mom1/mom2/mom3 of the box and
 * the new momentum of the interior.  fv: face velocity (the average of two
 * faces when staggered). */
static void swpzmom(const mc_ctx* m, int staggered, const double* fv, const double* c, int d, double* mom,
                    double* m1a, double* m2a, double* m3a) {
    og_grid* g = m->g;
    const long st3[3] = {1, g->sy, g->sz};
    const long o = st3[d];
    const double rho1 = m->rho1, rho2 = m->rho2, dt = m->dt, dxyz = m->dxyz;
    BOX_LOOP(g) {
        const long n = OG_IX(g, i, j, k);
        double a1, a2, uadv1 = 0.0, uadv3 = 0.0, uavg, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        if (staggered) {
            a2 = fv[n] * dt / dxyz;
            a1 = fv[n - o] * dt / dxyz;
            const double ro1 = (rho2 * c[n - o] + rho1 * (1.0 - c[n - o]));
            const double ro2 = (rho2 * c[n] + rho1 * (1.0 - c[n]));
            const double ro3 = (rho2 * c[n + o] + rho1 * (1.0 - c[n + o]));
            u1 = mom[n - o] / ro1;
            u2 = mom[n] / ro2;
            u3 = mom[n + o] / ro3;
            uadv1 = interpole3(u1, u2, u3, m->scheme, -0.5 - a1 / 2.0);
            uadv3 = interpole3(u1, u2, u3, m->scheme, 0.5 - a2 / 2.0);
        } else {
            a2 = fv[n] * dt / g->dxh[i];   /* dxh(i) of the x index, as the reference writes it */
            a1 = fv[n - o] * dt / dxyz;
        }
        const double mm1 = og_dmax1(a1, 0.0);
        const double mm2 = 1.0 - mm1 + og_dmin1(0.0, a2);
        if (staggered)
            uavg = interpole3(u1, u2, u3, m->scheme, (-og_dmin1(a1, 0.0) - og_dmax1(a2, 0.0)) / 2.0);
        else
            uavg = mom[n] / (rho2 * c[n] + rho1 * (1.0 - c[n]));
        m1a[n] = 0.0; m2a[n] = 0.0; m3a[n] = 0.0;
        if (c[n] > 0.0 && c[n] < 1.0) {
            double s[27], nr[3], alpha, vof, x0[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0};
            og_stencil(g, c, n, s);
            if (og_fit_plane_new(c[n], d, a1, a2, s, nr, &alpha)) continue;
            if (staggered && m->lin) {
                double sc[27], nrc[3], alphac, xcm1[3], xcm2[3];
                for (int q = 0; q < 27; q++) sc[q] = 1.0 - s[q];
                if (og_fit_plane_new(1.0 - c[n], d, a1, a2, sc, nrc, &alphac)) {
                    nrc[0] = -nr[0]; nrc[1] = -nr[1]; nrc[2] = -nr[2];
                    alphac = -alpha;
                }
                if (a1 < 0.0) {
                    uadv1 = interpole3(u1, u2, u3, m->scheme, -0.5 - a1 / 2.0 / (1.0 - a1 + a2));
                    uadv3 = interpole3(u1, u2, u3, m->scheme, -0.5);
                    x0[d] = a1;
                    dx[d] = -a1;
                    vof = og_fl3d(nr, alpha, x0, dx);
                    og_flux_centroid(nr, alpha, x0, dx, xcm1);
                    og_flux_centroid(nrc, alphac, x0, dx, xcm2);
                    m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1 +
                             (rho2 * vof * xcm1[d] + rho1 * (-a1 - vof) * xcm2[d]) * (uadv3 - uadv1) / a1;
                }
                if (a2 > 0.0) {
                    uadv1 = interpole3(u1, u2, u3, m->scheme, 0.5 - a2 / (1.0 - a1 + a2));
                    uadv3 = interpole3(u1, u2, u3, m->scheme, 0.5);
                    x0[d] = 1.0;
                    dx[d] = a2;
                    vof = og_fl3d(nr, alpha, x0, dx);
                    og_flux_centroid(nr, alpha, x0, dx, xcm1);
                    og_flux_centroid(nrc, alphac, x0, dx, xcm2);
                    m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * uadv1 +
                             (rho2 * (xcm1[d] - 1.0) * vof + rho1 * (xcm2[d] - 1.0) * (a2 - vof)) * (uadv3 - uadv1) / a2;
                }
                uadv1 = interpole3(u1, u2, u3, m->scheme, -0.5 - og_dmin1(a1, 0.0));
                uadv3 = interpole3(u1, u2, u3, m->scheme, 0.5 - og_dmax1(a2, 0.0));
                x0[d] = mm1;
                dx[d] = mm2;
                vof = og_fl3d(nr, alpha, x0, dx);
                og_flux_centroid(nr, alpha, x0, dx, xcm1);
                og_flux_centroid(nrc, alphac, x0, dx, xcm2);
                m2a[n] = (rho2 * vof + rho1 * (mm2 - vof)) * uadv1 +
                         (rho2 * (xcm1[d] - x0[d]) * vof + rho1 * (xcm2[d] - x0[d]) * (mm2 - vof)) * (uadv3 - uadv1) /
                             mm2;
            } else {
                const double w1 = staggered ? uadv1 : uavg, w3 = staggered ? uadv3 : uavg;
                if (a1 < 0.0) {
                    x0[d] = a1;
                    dx[d] = -a1;
                    vof = og_fl3d(nr, alpha, x0, dx);
                    m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * w1;
                }
                if (a2 > 0.0) {
                    x0[d] = 1.0;
                    dx[d] = a2;
                    vof = og_fl3d(nr, alpha, x0, dx);
                    m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * w3;
                }
                x0[d] = mm1;
                dx[d] = mm2;
                vof = og_fl3d(nr, alpha, x0, dx);
                m2a[n] = (rho2 * vof + rho1 * (mm2 - vof)) * uavg;
            }
        } else {
            const double w1 = staggered ? uadv1 : uavg, w3 = staggered ? uadv3 : uavg;
            double vof;
            if (a1 < 0.0) {
                vof = c[n] * (-a1);
                m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * w1;
            }
            if (a2 > 0.0) {
                vof = c[n] * a2;
                m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * w3;
            }
            vof = c[n] * mm2;
            m2a[n] = (rho2 * vof + rho1 * (mm2 - vof)) * uavg;
        }
    }
    INT_LOOP(g) {
        const long n = OG_IX(g, i, j, k);
        mom[n] = m1a[n + o] + m2a[n] + m3a[n - o];
    }
}

/* swprmom_stg (staggered = 1, vofnonmodule.f90:966-1139) or swprmom
 * (staggered = 0, :856-962): Weymouth-Yue fluxes mom1/mom3 and the update
 * with the central term of cg (c_mask of the volume fraction). */
static void swprmom(const mc_ctx* m, int staggered, const double* fv, const double* c, const double* cg, int d,
                    double* mom, double* m1a, double* m3a) {
    og_grid* g = m->g;
    const long st3[3] = {1, g->sy, g->sz};
    const long o = st3[d];
    const double rho1 = m->rho1, rho2 = m->rho2, dt = m->dt, dxyz = m->dxyz;
    BOX_LOOP(g) {
        const long n = OG_IX(g, i, j, k);
        m1a[n] = 0.0;
        m3a[n] = 0.0;
        const double a2 = fv[n] * dt / dxyz;
        const double a1 = fv[n - o] * dt / dxyz;
        double uadv1, uadv3, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        if (staggered) {
            const double ro1 = (rho2 * c[n - o] + rho1 * (1.0 - c[n - o]));
            const double ro2 = (rho2 * c[n] + rho1 * (1.0 - c[n]));
            const double ro3 = (rho2 * c[n + o] + rho1 * (1.0 - c[n + o]));
            u1 = mom[n - o] / ro1;
            u2 = mom[n] / ro2;
            u3 = mom[n + o] / ro3;
            uadv1 = interpole3(u1, u2, u3, m->scheme, -0.5 * (1.0 + a1));
            uadv3 = interpole3(u1, u2, u3, m->scheme, 0.5 * (1.0 - a2));
        } else {
            uadv1 = uadv3 = mom[n] / (rho2 * c[n] + rho1 * (1.0 - c[n]));
        }
        if (c[n] > 0.0 && c[n] < 1.0) {
            double s[27], mx[3], x0[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0}, vof;
            og_stencil(g, c, n, s);
            og_mycs(s, mx);
            const double alpha = og_al3d(mx, c[n]);
            if (staggered && m->lin) {
                double xcm1[3], xcm2[3];
                if (a1 < 0.0) {
                    uadv1 = interpole3(u1, u2, u3, m->scheme, -0.5);
                    uadv3 = interpole3(u1, u2, u3, m->scheme, -0.5 - a1);
                    dx[d] = -a1;
                    vof = og_fl3d(mx, alpha, x0, dx);
                    og_flux_centroid(mx, alpha, x0, dx, xcm1);
                    og_flux_centroid(mx, 1.0 - alpha, x0, dx, xcm2);
                    m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1 +
                             (rho2 * vof * xcm1[d] + rho1 * (-a1 - vof) * xcm2[d]) * (uadv3 - uadv1) / (-a1);
                }
                if (a2 > 0.0) {
                    uadv1 = interpole3(u1, u2, u3, m->scheme, 0.5 - a2);
                    uadv3 = interpole3(u1, u2, u3, m->scheme, 0.5);
                    x0[d] = 1.0 - a2;
                    dx[d] = a2;
                    vof = og_fl3d(mx, alpha, x0, dx);
                    og_flux_centroid(mx, 1.0 - alpha, x0, dx, xcm2);
                    og_flux_centroid(mx, alpha, x0, dx, xcm1);
                    m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * uadv1 +
                             (rho2 * vof * (xcm1[d] - x0[d]) + rho1 * (a2 - vof) * (xcm2[d] - x0[d])) *
                                 (uadv3 - uadv1) / a2;
                }
            } else {
                if (a1 < 0.0) {
                    dx[d] = -a1;
                    vof = og_fl3d(mx, alpha, x0, dx);
                    m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1;
                }
                if (a2 > 0.0) {
                    x0[d] = 1.0 - a2;
                    dx[d] = a2;
                    vof = og_fl3d(mx, alpha, x0, dx);
                    m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * uadv3;
                }
            }
        } else {
            double vof;
            if (a1 < 0.0) {
                vof = -a1 * c[n];
                m1a[n] = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1;
            }
            if (a2 > 0.0) {
                vof = a2 * c[n];
                m3a[n] = (rho2 * vof + rho1 * (a2 - vof)) * uadv3;
            }
        }
    }
    INT_LOOP(g) {
        const long n = OG_IX(g, i, j, k);
        const double a2 = fv[n] * dt / dxyz;
        const double a1 = fv[n - o] * dt / dxyz;
        const double uavg = mom[n] / (rho2 * c[n] + rho1 * (1.0 - c[n]));
        if (staggered)
            mom[n] = mom[n] - (m3a[n] - m1a[n + o]) + (m3a[n - o] - m1a[n]) + (rho2 - rho1) * cg[n] * uavg * (a2 - a1);
        else
            mom[n] = mom[n] - (m3a[n] - m1a[n + o]) + (m3a[n - o] - m1a[n]) +
                     (rho2 * cg[n] + rho1 * (1.0 - cg[n])) * uavg * (a2 - a1);
    }
}

/* SetMomentumBC then do_all_ghost(mom) after the sweep along d of component
 * dir: swpmom_stg passes d to SetMomentumBC from swpzmom_stg; swprmom_stg
 * passes dir when dir == 1 or d is 2 or 3, and skips it otherwise
 * (vofnonmodule.f90:620-629, :1128-1137); the centred sweeps pass d
 * (:420-429, :951-960). */
static void sweep_bc(const mc_ctx* m, int staggered, int wy, const double* us, const double* c, double* mom, int d,
                     int dir) {
    if (!staggered || !wy) set_momentum_bc(m, us, c, mom, d);
    else if (dir == 0 || d == 1 || d == 2) set_momentum_bc(m, us, c, mom, dir);
    og_do_all_ghost(m->g, mom);
}

int og_vof_mom_sweeps(const paris_grid_desc* desc, int tswap, double dt, int staggered, int lin_interp, int scheme,
                      const double* wallvel, const double* cvof, const int32_t* vof_flag, double* u, double* v,
                      double* w, double* du, double* dv, double* dw, double* mom) {
    for (int f = 0; f < 6; f++)
        if (desc->bdry_cond[f] != PARIS_BC_WALL && desc->bdry_cond[f] != PARIS_BC_PERIODIC) return PARIS_BAD_ARGS;
    og_grid* g = og_grid_new(desc);
    if (!g) return PARIS_BAD_ARGS;
    mc_ctx m;
    m.g = g;
    m.dt = dt;
    m.dxyz = g->dxh[g->ng];
    m.rho1 = desc->rho1;
    m.rho2 = desc->rho2;
    m.scheme = scheme;
    m.lin = lin_interp;
    for (int q = 0; q < 18; q++) m.wv[q] = wallvel ? wallvel[q] : 0.0;
    const long nt = g->ntot;
    const int wy = desc->vof_advect == PARIS_ADVECT_WY;
    double* tmp = malloc(nt * sizeof(double));
    double* w1 = calloc(nt, sizeof(double));
    double* w2 = calloc(nt, sizeof(double));
    double* w3 = calloc(nt, sizeof(double));
    double* fv = calloc(nt, sizeof(double));
    double* cg = calloc(nt, sizeof(double));
    int32_t* tflag = malloc(nt * sizeof(int32_t));
    double* vel[3] = {u, v, w};
    double* der[3] = {du, dv, dw};
    const long st3[3] = {1, g->sy, g->sz};
    int order[3];
    if (tswap % 3 == 0) { order[0] = 2; order[1] = 0; order[2] = 1; }
    else if (tswap % 3 == 1) { order[0] = 1; order[1] = 2; order[2] = 0; }
    else { order[0] = 0; order[1] = 1; order[2] = 2; }
    for (int dir = 0; dir < 3; dir++) {
        double* us = vel[dir];
        const long o2 = st3[dir];
        memcpy(tmp, cvof, nt * sizeof(double));
        memset(w1, 0, nt * sizeof(double));
        memset(w2, 0, nt * sizeof(double));
        if (staggered) {   /* get_momentum_staggered */
            BOX_LOOP(g) half_fractions(g, cvof, OG_IX(g, i, j, k), dir, &w1[OG_IX(g, i, j, k)], &w2[OG_IX(g, i, j, k)]);
            og_do_all_ghost(g, w1);
            og_do_all_ghost(g, w2);
            og_do_all_ghost(g, us);
            BOX_LOOP(g) {
                const long n = OG_IX(g, i, j, k);
                tmp[n] = og_dmax1(0.0, og_dmin1(1.0, 0.5 * (w2[n] + w1[n + o2])));
                const double rhoavg = tmp[n] * m.rho2 + (1.0 - tmp[n]) * m.rho1;
                mom[n] = us[n] * rhoavg;
            }
            set_momentum_bc(&m, us, cvof, mom, dir);
        } else {   /* get_momentum_centered */
            og_do_all_ghost(g, us);
            BOX_LOOP(g) {
                const long n = OG_IX(g, i, j, k);
                const double rhoavg = tmp[n] * m.rho2 + (1.0 - tmp[n]) * m.rho1;
                mom[n] = 0.5 * (us[n] + us[n - o2]) * rhoavg;
            }
        }
        og_do_all_ghost(g, tmp);
        og_do_all_ghost(g, mom);
        memcpy(tflag, vof_flag, nt * sizeof(int32_t));
        if (wy)   /* c_mask(tmp, work(:,:,:,2)) */
            for (long n = 0; n < nt; n++) cg[n] = tmp[n] > 0.5 ? 1.0 : 0.0;
        for (int s = 0; s < 3; s++) {
            const int d = order[s];
            const double* ud = vel[d];
            const double* face = ud;
            if (staggered) {   /* 0.5*(us(i) + us(i+e_dir)) of swpz_stg / swpr_stg */
                for (long n = 0; n < nt; n++) fv[n] = n + o2 < nt ? 0.5 * (ud[n] + ud[n + o2]) : 0.0;
                face = fv;
            }
            if (wy) swprmom(&m, staggered, face, tmp, cg, d, mom, w1, w3);
            else swpzmom(&m, staggered, face, tmp, d, mom, w1, w2, w3);
            sweep_bc(&m, staggered, wy, ud, tmp, mom, d, dir);
            og_swp(g, face, tmp, tflag, d, dt, w1, wy ? cg : w2, w3, NULL);
        }
        double* dd = der[dir];
        if (staggered) {   /* get_velocity_from_momentum_staggered */
            int iend = g->ng + g->nx - 1, jend = g->ng + g->ny - 1, kend = g->ng + g->nz - 1;
            if (dir == 0 && !og_is_periodic(g, 0)) iend--;
            if (dir == 1 && !og_is_periodic(g, 1)) jend--;
            if (dir == 2 && !og_is_periodic(g, 2)) kend--;
            for (int k = g->ng; k <= kend; k++)
                for (int j = g->ng; j <= jend; j++)
                    for (int i = g->ng; i <= iend; i++) {
                        const long n = OG_IX(g, i, j, k);
                        const double cflag = tmp[n];
                        if (cflag > 0.0 && cflag < 1.0) {
                            const double rhoavg = m.rho2 * cflag + (1.0 - cflag) * m.rho1;
                            dd[n] = (mom[n] / rhoavg - us[n]) / dt;
                        }
                    }
        } else {   /* get_velocity_from_momentum_centered */
            BOX_LOOP(g) {
                const long n = OG_IX(g, i, j, k);
                const double cf0 = tmp[n], cf1 = tmp[n + o2];
                const double r0 = m.rho2 * cf0 + (1.0 - cf0) * m.rho1;
                const double r1 = m.rho2 * cf1 + (1.0 - cf1) * m.rho1;
                if ((cf0 > 0.0 && cf0 < 1.0) || (cf1 > 0.0 && cf1 < 1.0))
                    dd[n] = ((mom[n] / r0 + mom[n + o2] / r1) * 0.5 - us[n]) / dt;
            }
        }
        og_do_all_ghost(g, dd);
    }
    free(tmp); free(w1); free(w2); free(w3); free(fv); free(cg); free(tflag);
    og_grid_free(g);
    return PARIS_OK;
}
