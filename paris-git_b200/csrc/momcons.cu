// momcons.cu -- the momentum-conserving VOF sweeps of DoMOMCONS on the
// device: vofandmomsweepsstaggered (vofmodules.f90:1536-1692).  For each
// velocity component dir:
//   1. the momentum on the control volume of that component and the volume
//      fraction of the control volume (get_momentum_staggered :1396-1449 with
//      get_half_fractions :1307-1338, or get_momentum_centered :1363-1394),
//      with SetMomentumBC (modules.f90:1329-1625) and the ghosts;
//   2. per split direction d in the order of MOD(tswap,3): the momentum
//      fluxes of the CIAM (swpzmom_stg vofnonmodule.f90:433-631, swpzmom
//      :333-431) or Weymouth-Yue (swprmom_stg :966-1139, swprmom :856-962)
//      sweep from the fraction before the sweep, the momentum update,
//      SetMomentumBC and the ghosts, then the split sweep of the fraction
//      itself (swp_stg :50-71 / swp), run by the VOF sweep kernels with the
//      face velocity of the control volume (0.5*(us(i) + us(i+e_dir)) for
//      the staggered volumes, formed into an array by the same operations);
//   3. du/dv/dw replaced by (mom/rho - u)/dt where the advected fraction is
//      mixed (get_velocity_from_momentum_staggered :1486-1534 /
//      get_velocity_from_momentum_centered :1451-1484), then the ghosts.
//
// One thread per cell throughout; the flux kernels cover the cells whose
// fluxes reach the interior (the interior across d, one cell beyond it along
// d), like the VOF sweeps.  Built with -fmad=false so that each expression
// keeps the Fortran operation order.
//
// Values the reference reads without setting are made definite: the
// momentum array starts at zero and keeps the ghost cells no loop or
// boundary condition writes; with LinInterp a failed complementary plane fit
// takes the complement of the cell's own plane (-nr, -alpha).  The solid mask
// of SetMomentumBC is 1 everywhere (no obstacles) and is left out.  The
// staggered fraction, the mean of two half-cell fractions, is clipped to
// [0, 1]: a half fraction of a nearly full cell can round to just above 1,
// and a fraction above 1 sends AL3D into the cube root of a negative number
// (NaN); the reference does not clip and depends on that rounding.
#include <cmath>

#include "ctx.cuh"
#include "limiter.cuh"
#include "plic.cuh"

namespace {

struct WallV {
    double v[18];   // WallVel(f, c) at (f-1) + 6 (c-1)
};

struct McArgs {
    const double* c;      // the advected fraction before this sweep
    double* mom;
    const double* fv;     // face velocity of the sweep along d
    const uint8_t* cg;    // c_mask of the fraction (Weymouth-Yue)
    double *m1, *m2, *m3; // momentum fluxes mom1 / mom2 / mom3
    const double* dxh;    // dxh by x index + ng
    Layout L;
    int d, scheme;
    double dt, dxyz, rho1, rho2;
};

__host__ __device__ inline long dstride(const Layout& L, int d) { return d == 0 ? 1 : (d == 1 ? L.pitch : L.plane); }

// (i, j, k), interior-relative, of a flux cell: the interior across d,
// -1 .. n along d
__device__ inline bool flux_cell(const Layout& L, int d, int& i, int& j, int& k) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y;
    k = blockIdx.z;
    if (d == 0) i -= 1; else if (d == 1) j -= 1; else k -= 1;
    return i <= L.n[0] && (d == 0 || i < L.n[0]);
}

// (i, j, k), interior-relative, of element t of the ghosted array
__device__ inline void cell_of(const Layout& L, long t, int& i, int& j, int& k) {
    const long rows = L.plane / L.pitch;
    i = (int)(t % L.pitch) - L.ng;
    j = (int)((t / L.pitch) % rows) - L.ng;
    k = (int)(t / L.plane) - L.ng;
}

__device__ inline bool in_box(const Layout& L, int i, int j, int k) {   // [is-1, ie+1]^3
    return i >= -1 && j >= -1 && k >= -1 && i <= L.n[0] && j <= L.n[1] && k <= L.n[2];
}

__device__ inline void stencil(const double* __restrict__ c, const Layout& L, long n, double st[27]) {
#pragma unroll
    for (int k1 = -1; k1 <= 1; k1++)
#pragma unroll
        for (int j1 = -1; j1 <= 1; j1++)
#pragma unroll
            for (int i1 = -1; i1 <= 1; i1++)
                st[(i1 + 1) + 3 * (j1 + 1) + 9 * (k1 + 1)] = c[n + i1 + j1 * L.pitch + k1 * L.plane];
}

// fit_plane_new, vofnonmodule.f90:633-655; false on a zero normal
__device__ inline bool fit_plane_new(double vof, int d, double a1, double a2, const double st[27], double m[3],
                                     double& alpha) {
    plic::mycs(st, m);
    if (m[0] == 0.0 && m[1] == 0.0 && m[2] == 0.0) return false;
    alpha = plic::al3d(m, vof);
    m[d] = m[d] / (1.0 - a1 + a2);
    alpha = alpha + m[d] * a1;
    return true;
}

__device__ inline double rho_of(double rho1, double rho2, double c) { return rho2 * c + rho1 * (1.0 - c); }

// The PLIC geometry of the sweeps works on a plane held as four scalars,
// and every helper that builds a local array (the 3x3x3 stencil, the normal,
// the flux box) is a separate, non-inlined function with its own frame: in
// the large flux kernels, inlined helpers with address-taken local arrays
// were seen to read back values that no statement of theirs wrote.
struct Plane {
    double n0, n1, n2, alpha;
};

// fit_plane_new (vofnonmodule.f90:633-655) of cell n, on the stencil of c or
// (complement) of 1 - c; false on a zero normal
__device__ __noinline__ bool mc_fit_plane(const double* __restrict__ c, const Layout L, long n, int d, double a1,
                                          double a2, int complement, Plane* P) {
    double st[27], m[3], alpha;
    stencil(c, L, n, st);
    double vof = c[n];
    if (complement) {
        for (int q = 0; q < 27; q++) st[q] = 1.0 - st[q];
        vof = 1.0 - vof;
    }
    if (!fit_plane_new(vof, d, a1, a2, st, m, alpha)) return false;
    P->n0 = m[0];
    P->n1 = m[1];
    P->n2 = m[2];
    P->alpha = alpha;
    return true;
}

// mycs + AL3D of cell n (swpr / swprmom: no mapping, no zero-normal check)
__device__ __noinline__ void mc_plane_wy(const double* __restrict__ c, const Layout L, long n, Plane* P) {
    double st[27], m[3];
    stencil(c, L, n, st);
    plic::mycs(st, m);
    P->alpha = plic::al3d(m, c[n]);
    P->n0 = m[0];
    P->n1 = m[1];
    P->n2 = m[2];
}

// FL3D and the d-component of FLUX_CENTROID of the plane in the unit box cut
// to [lo, lo + len] along d (x0 = lo e_d, dx = 1 + (len - 1) e_d), the boxes
// the sweeps build by setting x0(d) and deltax(d)
__device__ __noinline__ double fl3d_seg(const Plane P, int d, double lo, double len) {
    const double nr[3] = {P.n0, P.n1, P.n2};
    const double x0[3] = {d == 0 ? lo : 0.0, d == 1 ? lo : 0.0, d == 2 ? lo : 0.0};
    const double dx[3] = {d == 0 ? len : 1.0, d == 1 ? len : 1.0, d == 2 ? len : 1.0};
    return plic::fl3d(nr, P.alpha, x0, dx);
}
__device__ __noinline__ double centroid_seg(const Plane P, int d, double lo, double len) {
    const double nr[3] = {P.n0, P.n1, P.n2};
    const double x0[3] = {d == 0 ? lo : 0.0, d == 1 ? lo : 0.0, d == 2 ? lo : 0.0};
    const double dx[3] = {d == 0 ? len : 1.0, d == 1 ? len : 1.0, d == 2 ? len : 1.0};
    double xc[3];
    plic::flux_centroid(nr, P.alpha, x0, dx, xc);
    return d == 0 ? xc[0] : (d == 1 ? xc[1] : xc[2]);
}

// get_half_fractions of cvof along dir into w1 (lower half) and w2 (upper
// half) over the [is-1, ie+1] box, zero elsewhere
__global__ void k_mc_half(const double* __restrict__ c, double* __restrict__ w1, double* __restrict__ w2,
                          const Layout L, int dir) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= L.total) return;
    int i, j, k;
    cell_of(L, t, i, j, k);
    double h1 = 0.0, h2 = 0.0;
    if (in_box(L, i, j, k)) {
        const double cc = c[t];
        h1 = cc;
        h2 = cc;
        if (cc > 0.0 && cc < 1.0) {
            Plane P;
            if (mc_fit_plane(c, L, t, dir, 0.0, 0.0, 0, &P)) {
                h1 = 2.0 * fl3d_seg(P, dir, 0.0, 0.5);
                h2 = 2.0 * fl3d_seg(P, dir, 0.5, 0.5);
            }
        }
    }
    w1[t] = h1;
    w2[t] = h2;
}

// the fraction and momentum of the control volumes over the box; the
// fraction is cvof elsewhere, the momentum keeps its value elsewhere
__global__ void k_mc_momentum(const double* __restrict__ cvof, const double* __restrict__ w1,
                              const double* __restrict__ w2, const double* __restrict__ us, double* __restrict__ tmp,
                              double* __restrict__ mom, const Layout L, int dir, int staggered, double rho1,
                              double rho2) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= L.total) return;
    int i, j, k;
    cell_of(L, t, i, j, k);
    const long o2 = dstride(L, dir);
    double tv = cvof[t];
    if (in_box(L, i, j, k)) {
        if (staggered) {
            tv = plic::dmax1(0.0, plic::dmin1(1.0, 0.5 * (w2[t] + w1[t + o2])));
            const double rhoavg = tv * rho2 + (1.0 - tv) * rho1;
            mom[t] = us[t] * rhoavg;
        } else {
            const double rhoavg = tv * rho2 + (1.0 - tv) * rho1;
            mom[t] = 0.5 * (us[t] + us[t - o2]) * rhoavg;
        }
    }
    tmp[t] = tv;
}

// 0.5*(us(i) + us(i+e_dir)) wherever i+e_dir is in the array
__global__ void k_mc_face_avg(const double* __restrict__ us, double* __restrict__ fv, long o2, long total) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    fv[t] = t + o2 < total ? 0.5 * (us[t] + us[t + o2]) : 0.0;
}

// CIAM momentum fluxes of one flux cell: swpzmom_stg (STAG; LIN: LinInterp)
// or swpzmom
template <bool STAG, bool LIN>
__global__ void __launch_bounds__(128) k_mc_ciam_flux(const McArgs a) {
    int i, j, k;
    const Layout& L = a.L;
    if (!flux_cell(L, a.d, i, j, k)) return;
    const long n = lidx(L, i, j, k), o = dstride(L, a.d);
    const double* __restrict__ c = a.c;
    const double rho1 = a.rho1, rho2 = a.rho2;
    const int d = a.d;
    double a1, a2, uadv1 = 0.0, uadv3 = 0.0, uavg, u1 = 0.0, u2 = 0.0, u3 = 0.0;
    const double cc = c[n];
    if (STAG) {
        a2 = a.fv[n] * a.dt / a.dxyz;
        a1 = a.fv[n - o] * a.dt / a.dxyz;
        const double ro1 = (rho2 * c[n - o] + rho1 * (1.0 - c[n - o]));
        const double ro2 = (rho2 * cc + rho1 * (1.0 - cc));
        const double ro3 = (rho2 * c[n + o] + rho1 * (1.0 - c[n + o]));
        u1 = a.mom[n - o] / ro1;
        u2 = a.mom[n] / ro2;
        u3 = a.mom[n + o] / ro3;
        uadv1 = interpole3(u1, u2, u3, a.scheme, -0.5 - a1 / 2.0);
        uadv3 = interpole3(u1, u2, u3, a.scheme, 0.5 - a2 / 2.0);
    } else {
        a2 = a.fv[n] * a.dt / a.dxh[i + L.ng];   // dxh(i) of the x index, as the reference writes it
        a1 = a.fv[n - o] * a.dt / a.dxyz;
    }
    const double mm1 = plic::dmax1(a1, 0.0);
    const double mm2 = 1.0 - mm1 + plic::dmin1(0.0, a2);
    if (STAG) uavg = interpole3(u1, u2, u3, a.scheme, (-plic::dmin1(a1, 0.0) - plic::dmax1(a2, 0.0)) / 2.0);
    else uavg = a.mom[n] / (rho2 * cc + rho1 * (1.0 - cc));
    double f1 = 0.0, f2 = 0.0, f3 = 0.0;
    if (cc > 0.0 && cc < 1.0) {
        Plane P;
        double vof;
        if (mc_fit_plane(c, L, n, d, a1, a2, 0, &P)) {
            if (LIN) {
                Plane Q;
                if (!mc_fit_plane(c, L, n, d, a1, a2, 1, &Q)) Q = Plane{-P.n0, -P.n1, -P.n2, -P.alpha};
                if (a1 < 0.0) {
                    uadv1 = interpole3(u1, u2, u3, a.scheme, -0.5 - a1 / 2.0 / (1.0 - a1 + a2));
                    uadv3 = interpole3(u1, u2, u3, a.scheme, -0.5);
                    vof = fl3d_seg(P, d, a1, -a1);
                    const double xcm1 = centroid_seg(P, d, a1, -a1);
                    const double xcm2 = centroid_seg(Q, d, a1, -a1);
                    f1 = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1 +
                         (rho2 * vof * xcm1 + rho1 * (-a1 - vof) * xcm2) * (uadv3 - uadv1) / a1;
                }
                if (a2 > 0.0) {
                    uadv1 = interpole3(u1, u2, u3, a.scheme, 0.5 - a2 / (1.0 - a1 + a2));
                    uadv3 = interpole3(u1, u2, u3, a.scheme, 0.5);
                    vof = fl3d_seg(P, d, 1.0, a2);
                    const double xcm1 = centroid_seg(P, d, 1.0, a2);
                    const double xcm2 = centroid_seg(Q, d, 1.0, a2);
                    f3 = (rho2 * vof + rho1 * (a2 - vof)) * uadv1 +
                         (rho2 * (xcm1 - 1.0) * vof + rho1 * (xcm2 - 1.0) * (a2 - vof)) * (uadv3 - uadv1) / a2;
                }
                uadv1 = interpole3(u1, u2, u3, a.scheme, -0.5 - plic::dmin1(a1, 0.0));
                uadv3 = interpole3(u1, u2, u3, a.scheme, 0.5 - plic::dmax1(a2, 0.0));
                vof = fl3d_seg(P, d, mm1, mm2);
                const double xcm1 = centroid_seg(P, d, mm1, mm2);
                const double xcm2 = centroid_seg(Q, d, mm1, mm2);
                f2 = (rho2 * vof + rho1 * (mm2 - vof)) * uadv1 +
                     (rho2 * (xcm1 - mm1) * vof + rho1 * (xcm2 - mm1) * (mm2 - vof)) * (uadv3 - uadv1) / mm2;
            } else {
                const double w1 = STAG ? uadv1 : uavg, w3 = STAG ? uadv3 : uavg;
                if (a1 < 0.0) {
                    vof = fl3d_seg(P, d, a1, -a1);
                    f1 = (rho2 * vof + rho1 * (-a1 - vof)) * w1;
                }
                if (a2 > 0.0) {
                    vof = fl3d_seg(P, d, 1.0, a2);
                    f3 = (rho2 * vof + rho1 * (a2 - vof)) * w3;
                }
                vof = fl3d_seg(P, d, mm1, mm2);
                f2 = (rho2 * vof + rho1 * (mm2 - vof)) * uavg;
            }
        }
    } else {
        const double w1 = STAG ? uadv1 : uavg, w3 = STAG ? uadv3 : uavg;
        double vof;
        if (a1 < 0.0) {
            vof = cc * (-a1);
            f1 = (rho2 * vof + rho1 * (-a1 - vof)) * w1;
        }
        if (a2 > 0.0) {
            vof = cc * a2;
            f3 = (rho2 * vof + rho1 * (a2 - vof)) * w3;
        }
        vof = cc * mm2;
        f2 = (rho2 * vof + rho1 * (mm2 - vof)) * uavg;
    }
    a.m1[n] = f1;
    a.m2[n] = f2;
    a.m3[n] = f3;
}

// Weymouth-Yue momentum fluxes of one flux cell: swprmom_stg (STAG; LIN:
// LinInterp) or swprmom
template <bool STAG, bool LIN>
__global__ void __launch_bounds__(128) k_mc_wy_flux(const McArgs a) {
    int i, j, k;
    const Layout& L = a.L;
    if (!flux_cell(L, a.d, i, j, k)) return;
    const long n = lidx(L, i, j, k), o = dstride(L, a.d);
    const double* __restrict__ c = a.c;
    const double rho1 = a.rho1, rho2 = a.rho2;
    const int d = a.d;
    const double a2 = a.fv[n] * a.dt / a.dxyz;
    const double a1 = a.fv[n - o] * a.dt / a.dxyz;
    const double cc = c[n];
    double uadv1, uadv3, u1 = 0.0, u2 = 0.0, u3 = 0.0;
    if (STAG) {
        const double ro1 = (rho2 * c[n - o] + rho1 * (1.0 - c[n - o]));
        const double ro2 = (rho2 * cc + rho1 * (1.0 - cc));
        const double ro3 = (rho2 * c[n + o] + rho1 * (1.0 - c[n + o]));
        u1 = a.mom[n - o] / ro1;
        u2 = a.mom[n] / ro2;
        u3 = a.mom[n + o] / ro3;
        uadv1 = interpole3(u1, u2, u3, a.scheme, -0.5 * (1.0 + a1));
        uadv3 = interpole3(u1, u2, u3, a.scheme, 0.5 * (1.0 - a2));
    } else {
        uadv1 = uadv3 = a.mom[n] / (rho2 * cc + rho1 * (1.0 - cc));
    }
    double f1 = 0.0, f3 = 0.0;
    if (cc > 0.0 && cc < 1.0) {
        Plane P;
        double vof;
        mc_plane_wy(c, L, n, &P);
        const Plane Q{P.n0, P.n1, P.n2, 1.0 - P.alpha};   // flux_centroid(mxyz, 1 - alpha, ...)
        if (LIN) {
            if (a1 < 0.0) {
                uadv1 = interpole3(u1, u2, u3, a.scheme, -0.5);
                uadv3 = interpole3(u1, u2, u3, a.scheme, -0.5 - a1);
                vof = fl3d_seg(P, d, 0.0, -a1);
                const double xcm1 = centroid_seg(P, d, 0.0, -a1);
                const double xcm2 = centroid_seg(Q, d, 0.0, -a1);
                f1 = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1 +
                     (rho2 * vof * xcm1 + rho1 * (-a1 - vof) * xcm2) * (uadv3 - uadv1) / (-a1);
            }
            if (a2 > 0.0) {
                uadv1 = interpole3(u1, u2, u3, a.scheme, 0.5 - a2);
                uadv3 = interpole3(u1, u2, u3, a.scheme, 0.5);
                const double lo = 1.0 - a2;
                vof = fl3d_seg(P, d, lo, a2);
                const double xcm2 = centroid_seg(Q, d, lo, a2);
                const double xcm1 = centroid_seg(P, d, lo, a2);
                f3 = (rho2 * vof + rho1 * (a2 - vof)) * uadv1 +
                     (rho2 * vof * (xcm1 - lo) + rho1 * (a2 - vof) * (xcm2 - lo)) * (uadv3 - uadv1) / a2;
            }
        } else {
            if (a1 < 0.0) {
                vof = fl3d_seg(P, d, 0.0, -a1);
                f1 = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1;
            }
            if (a2 > 0.0) {
                vof = fl3d_seg(P, d, 1.0 - a2, a2);
                f3 = (rho2 * vof + rho1 * (a2 - vof)) * uadv3;
            }
        }
    } else {
        double vof;
        if (a1 < 0.0) {
            vof = -a1 * cc;
            f1 = (rho2 * vof + rho1 * (-a1 - vof)) * uadv1;
        }
        if (a2 > 0.0) {
            vof = a2 * cc;
            f3 = (rho2 * vof + rho1 * (a2 - vof)) * uadv3;
        }
    }
    a.m1[n] = f1;
    a.m3[n] = f3;
}

// the momentum of the interior after the sweep along d
template <bool WY, bool STAG>
__global__ void k_mc_update(const McArgs a) {
    const Layout& L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const long n = lidx(L, i, blockIdx.y, blockIdx.z), o = dstride(L, a.d);
    if (!WY) {
        a.mom[n] = a.m1[n + o] + a.m2[n] + a.m3[n - o];
    } else {
        const double a2 = a.fv[n] * a.dt / a.dxyz;
        const double a1 = a.fv[n - o] * a.dt / a.dxyz;
        const double cc = a.c[n], m0 = a.mom[n], cg = (double)a.cg[n];
        const double uavg = m0 / (a.rho2 * cc + a.rho1 * (1.0 - cc));
        if (STAG)
            a.mom[n] = m0 - (a.m3[n] - a.m1[n + o]) + (a.m3[n - o] - a.m1[n]) +
                       (a.rho2 - a.rho1) * cg * uavg * (a2 - a1);
        else
            a.mom[n] = m0 - (a.m3[n] - a.m1[n + o]) + (a.m3[n - o] - a.m1[n]) +
                       (a.rho2 * cg + a.rho1 * (1.0 - cg)) * uavg * (a2 - a1);
    }
}

// SetMomentumBC(u, c, mom, d, ...) on the wall faces normal to one axis, in
// the reference's order (x, then y, then z launches; low face, then high);
// each thread owns one line of the ghosted plane normal to the axis.  A wall
// normal to d gets mom = 0 on the face and the odd image behind it; the
// other walls get (2 WallVel - u) rho(c) from the first interior cell (on the
// x+ wall raised to the power rho(c), as the reference writes it).
__global__ void k_mc_wall_bc(double* __restrict__ mom, const double* __restrict__ u, const double* __restrict__ c,
                             const Layout L, int axis, int lo, int hi, int d, WallV WV, double rho1, double rho2) {
    const int g = L.ng;
    const int ta = axis == 0 ? 1 : 0, tb = axis == 2 ? 1 : 2;
    const int na = L.n[ta] + 2 * g, nb = L.n[tb] + 2 * g;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= na * nb) return;
    int q[3];
    q[ta] = p % na - g;
    q[tb] = p / na - g;
    const long s = dstride(L, axis);
    const int comp = axis == 0 ? 2 : 1;   // WallVel component of the tangential lines
    auto wv = [&](int f) { return WV.v[(f - 1) + 6 * (comp - 1)]; };
    if (lo) {
        q[axis] = 0;
        const long n0 = lidx(L, q[0], q[1], q[2]);
        if (d == axis) {
            mom[n0 - s] = 0.0;
            mom[n0 - 2 * s] = -mom[n0];
        } else {
            mom[n0 - s] = (2 * wv(2 * axis + 1) - u[n0]) * rho_of(rho1, rho2, c[n0]);
        }
    }
    if (hi) {
        q[axis] = L.n[axis] - 1;
        const long ne = lidx(L, q[0], q[1], q[2]);
        if (d == axis) {
            mom[ne] = 0.0;
            mom[ne + s] = -mom[ne - s];
        } else if (axis == 0) {
            mom[ne + s] = pow(2 * wv(2) - u[ne], rho_of(rho1, rho2, c[ne]));
        } else {
            mom[ne + s] = (2 * wv(2 * axis + 2) - u[ne]) * rho_of(rho1, rho2, c[ne]);
        }
    }
}

// get_velocity_from_momentum_staggered: the interior faces of component dir
// (is..ieu etc.) where the advected fraction is mixed
__global__ void k_mc_velocity_stg(const double* __restrict__ tmp, const double* __restrict__ mom,
                                  const double* __restrict__ us, double* __restrict__ der, const Layout L, int iend,
                                  int jend, int kend, double dt, double rho1, double rho2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= iend || j >= jend || k >= kend) return;
    const long n = lidx(L, i, j, k);
    const double cflag = tmp[n];
    if (cflag > 0.0 && cflag < 1.0) {
        const double rhoavg = rho2 * cflag + (1.0 - cflag) * rho1;
        der[n] = (mom[n] / rhoavg - us[n]) / dt;
    }
}

// get_velocity_from_momentum_centered: the [is-1, ie+1] box, the average of
// the two cell-centred velocities around the face
__global__ void k_mc_velocity_cen(const double* __restrict__ tmp, const double* __restrict__ mom,
                                  const double* __restrict__ us, double* __restrict__ der, const Layout L, int dir,
                                  double dt, double rho1, double rho2) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= L.total) return;
    int i, j, k;
    cell_of(L, t, i, j, k);
    if (!in_box(L, i, j, k)) return;
    const long o2 = dstride(L, dir);
    const double cf0 = tmp[t], cf1 = tmp[t + o2];
    const double r0 = rho2 * cf0 + (1.0 - cf0) * rho1;
    const double r1 = rho2 * cf1 + (1.0 - cf1) * rho1;
    if ((cf0 > 0.0 && cf0 < 1.0) || (cf1 > 0.0 && cf1 < 1.0))
        der[t] = ((mom[t] / r0 + mom[t + o2] / r1) * 0.5 - us[t]) / dt;
}

__global__ void k_mc_copy_i8(int8_t* __restrict__ dst, const int8_t* __restrict__ src, long total) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < total) dst[t] = src[t];
}

}  // namespace

// SetMomentumBC for the wall faces of the grid, then nothing else: the
// caller refreshes the ghosts
static int mc_wall_bc(paris_ctx* c, double* mom, const double* u, const double* cf, int d, const WallV& WV) {
    const Layout& L = c->L;
    for (int axis = 0; axis < 3; axis++) {
        const int lo = c->d.bdry_cond[axis] == PARIS_BC_WALL, hi = c->d.bdry_cond[axis + 3] == PARIS_BC_WALL;
        if (!lo && !hi) continue;
        const int ta = axis == 0 ? 1 : 0, tb = axis == 2 ? 1 : 2;
        const int lines = (L.n[ta] + 2 * L.ng) * (L.n[tb] + 2 * L.ng);
        PARIS_LAUNCH(c, k_mc_wall_bc, div_up(lines, 128), 128, 0, mom, u, cf, L, axis, lo, hi, d, WV, c->d.rho1,
                     c->d.rho2);
    }
    return PARIS_OK;
}

static int mc_alloc(paris_ctx* c) {
    const long nt = c->L.total;
    if (!c->mc_tmp) {
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_tmp, nt * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_tmp2, nt * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_work, 3 * nt * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_fv, nt * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_flag, nt));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mc_cg, nt));
        PARIS_CUDA_TRY(c, cudaMemsetAsync(c->mc_fv, 0, nt * sizeof(double), c->stream));
        PARIS_CUDA_TRY(c, cudaMemsetAsync(c->mc_tmp2, 0, nt * sizeof(double), c->stream));
    }
    return PARIS_OK;
}

extern "C" int paris_vof_mom_sweeps(paris_handle_t c, int32_t tswap, double dt, int32_t staggered,
                                    int32_t lin_interp, int32_t scheme, const double* wall_vel) {
    if (!c) return PARIS_BAD_ARGS;
    for (int f = 0; f < 6; f++)
        if (c->d.bdry_cond[f] != PARIS_BC_WALL && c->d.bdry_cond[f] != PARIS_BC_PERIODIC) {
            ctx_set_error(c, "vof_mom_sweeps: boundary type %d (periodic and walls only)", c->d.bdry_cond[f]);
            return PARIS_BAD_ARGS;
        }
    if (scheme < PARIS_CONV_QUICK || scheme > PARIS_CONV_WENO || !(dt > 0.0)) {
        ctx_set_error(c, "vof_mom_sweeps: scheme %d, dt %g", scheme, dt);
        return PARIS_BAD_ARGS;
    }
    const int g = c->d.ng;
    {
        const double hx = c->h_dxh[g], hy = c->h_dyh[g], hz = c->h_dzh[g];
        if (fabs(hy - hx) * 1e12 / hx > 1.0 || fabs(hz - hx) * 1e12 / hx > 1.0) {
            ctx_set_error(c, "vof_mom_sweeps: non-cubic cells");
            return PARIS_BAD_ARGS;
        }
    }
    cudaSetDevice(c->dev);
    for (int f : {PARIS_FIELD_CVOF, PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_DU, PARIS_FIELD_DV,
                  PARIS_FIELD_DW, PARIS_FIELD_MOMENTUM})
        PARIS_CHECK(ctx_alloc_field(c, f));
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_VOF_FLAG));
    PARIS_CHECK(mc_alloc(c));
    const Layout& L = c->L;
    const long nt = L.total;
    WallV WV;
    for (int q = 0; q < 18; q++) WV.v[q] = wall_vel ? wall_vel[q] : 0.0;
    const int wy = c->d.vof_advect == PARIS_ADVECT_WY;
    double* mom = c->fld[PARIS_FIELD_MOMENTUM];
    const double* cvof = c->fld[PARIS_FIELD_CVOF];
    double* w1 = c->mc_work;
    double* w2 = c->mc_work + nt;
    double* w3 = c->mc_work + 2 * nt;
    int order[3];
    const int m = ((tswap % 3) + 3) % 3;
    if (m == 0) { order[0] = 2; order[1] = 0; order[2] = 1; }
    else if (m == 1) { order[0] = 1; order[1] = 2; order[2] = 0; }
    else { order[0] = 0; order[1] = 1; order[2] = 2; }
    const unsigned gb = (unsigned)div_up(nt, 256L);
    for (int dir = 0; dir < 3; dir++) {
        double* us = c->fld[PARIS_FIELD_U + dir];
        double* tmp = c->mc_tmp;
        // 1. the control volumes: fraction and momentum
        if (staggered) {
            PARIS_LAUNCH_N(c, "mc_half_fractions", nt, k_mc_half, gb, 256, 0, cvof, w1, w2, L, dir);
            PARIS_CHECK(ctx_ghost_fill(c, w1));
            PARIS_CHECK(ctx_ghost_fill(c, w2));
        }
        PARIS_CHECK(ctx_ghost_fill(c, us));
        PARIS_LAUNCH_N(c, "mc_momentum", nt, k_mc_momentum, gb, 256, 0, cvof, w1, w2, us, tmp, mom, L, dir,
                       staggered, c->d.rho1, c->d.rho2);
        if (staggered) PARIS_CHECK(mc_wall_bc(c, mom, us, cvof, dir, WV));
        PARIS_CHECK(ctx_ghost_fill(c, tmp));
        PARIS_CHECK(ctx_ghost_fill(c, mom));
        PARIS_LAUNCH(c, k_mc_copy_i8, gb, 256, 0, c->mc_flag, c->flag, nt);
        if (wy) PARIS_LAUNCH(c, k_c_mask, gb, 256, 0, tmp, c->mc_cg, nt);
        // 2. the three split sweeps of momentum and fraction
        for (int s = 0; s < 3; s++) {
            const int d = order[s];
            const double* ud = c->fld[PARIS_FIELD_U + d];
            const double* face = ud;
            if (staggered) {
                PARIS_LAUNCH(c, k_mc_face_avg, gb, 256, 0, ud, c->mc_fv, dstride(L, dir), nt);
                face = c->mc_fv;
            }
            McArgs a;
            a.c = tmp;
            a.mom = mom;
            a.fv = face;
            a.cg = c->mc_cg;
            a.m1 = w1;
            a.m2 = w2;
            a.m3 = w3;
            a.dxh = c->dxh;
            a.L = L;
            a.d = d;
            a.scheme = scheme;
            a.dt = dt;
            a.dxyz = c->h_dxh[g];
            a.rho1 = c->d.rho1;
            a.rho2 = c->d.rho2;
            int ext[3] = {L.n[0], L.n[1], L.n[2]};
            ext[d] += 2;
            const dim3 fg(div_up(ext[0], 128), ext[1], ext[2]), ig(div_up(L.n[0], 128), L.n[1], L.n[2]);
            if (wy) {
                if (staggered && lin_interp) PARIS_LAUNCH_N(c, "mc_wy_flux", c->N, (k_mc_wy_flux<true, true>), fg, 128, 0, a);
                else if (staggered) PARIS_LAUNCH_N(c, "mc_wy_flux", c->N, (k_mc_wy_flux<true, false>), fg, 128, 0, a);
                else PARIS_LAUNCH_N(c, "mc_wy_flux", c->N, (k_mc_wy_flux<false, false>), fg, 128, 0, a);
                if (staggered) PARIS_LAUNCH_N(c, "mc_update", c->N, (k_mc_update<true, true>), ig, 128, 0, a);
                else PARIS_LAUNCH_N(c, "mc_update", c->N, (k_mc_update<true, false>), ig, 128, 0, a);
            } else {
                if (staggered && lin_interp)
                    PARIS_LAUNCH_N(c, "mc_ciam_flux", c->N, (k_mc_ciam_flux<true, true>), fg, 128, 0, a);
                else if (staggered) PARIS_LAUNCH_N(c, "mc_ciam_flux", c->N, (k_mc_ciam_flux<true, false>), fg, 128, 0, a);
                else PARIS_LAUNCH_N(c, "mc_ciam_flux", c->N, (k_mc_ciam_flux<false, false>), fg, 128, 0, a);
                PARIS_LAUNCH_N(c, "mc_update", c->N, (k_mc_update<false, false>), ig, 128, 0, a);
            }
            // SetMomentumBC after the sweep (the momentum of component d for
            // the CIAM and centred sweeps; swprmom_stg passes dir when dir is
            // x or d is y or z, and none otherwise), then do_all_ghost(mom)
            if (!staggered || !wy) PARIS_CHECK(mc_wall_bc(c, mom, ud, tmp, d, WV));
            else if (dir == 0 || d == 1 || d == 2) PARIS_CHECK(mc_wall_bc(c, mom, ud, tmp, dir, WV));
            PARIS_CHECK(ctx_ghost_fill(c, mom));
            // the split sweep of the fraction with the same face velocity
            PARIS_CHECK(vof_sweep_dir(c, d, dt, tmp, c->mc_tmp2, c->mc_flag, face, c->mc_cg));
            c->mc_tmp = c->mc_tmp2;
            c->mc_tmp2 = tmp;
            tmp = c->mc_tmp;
        }
        // 3. du/dv/dw where the advected fraction is mixed
        double* der = c->fld[PARIS_FIELD_DU + dir];
        if (staggered) {
            int end[3] = {L.n[0], L.n[1], L.n[2]};
            if (!c->bnd.per[dir]) end[dir] -= 1;
            PARIS_LAUNCH_N(c, "mc_velocity", c->N, k_mc_velocity_stg, dim3(div_up(end[0], 128), end[1], end[2]), 128,
                           0, tmp, mom, us, der, L, end[0], end[1], end[2], dt, c->d.rho1, c->d.rho2);
        } else {
            PARIS_LAUNCH_N(c, "mc_velocity", c->N, k_mc_velocity_cen, gb, 256, 0, tmp, mom, us, der, L, dir, dt,
                           c->d.rho1, c->d.rho2);
        }
        PARIS_CHECK(ctx_ghost_fill(c, der));
    }
    return PARIS_OK;
}
