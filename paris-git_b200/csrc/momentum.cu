// momentum.cu -- the explicit momentum predictor on the device:
// momentumConvection (paris.f90:1957-1984) with the QUICK scheme
// (momentumConvectionQUICK, paris.f90:2288-2414) or the one-dimensional
// ENO / Superbee / WENO schemes (momentumConvection_onedim,
// paris.f90:1991-2071; slope_lim, modules.f90:177-197), explicitMomDiff
// (paris.f90:2757-2808), volumeForce (paris.f90:2813-2860), u = u + dt*du
// (paris.f90:442-444) and the wall / periodic part of SetVelocityBC
// (modules.f90:951-973,1061-1105) with do_ghost_vector.
//
// Built with -fmad=false: each expression keeps the Fortran operation
// order, so results equal the FP64 restatement bit for bit.  The face values
// the reference keeps in its `work` array are recomputed where they are used
// (same operands, same operations), one thread per cell.
#include "ctx.cuh"

namespace {

struct Ax {   // one axis: cell centres, face positions, cell widths, centre spacings (index i+ng)
    const double *c, *h, *d, *dh;
};
struct Geo {
    Ax a[3];
};
struct Vel {
    const double *u, *v, *w;
};

// inter(x0,x1,x2,x,y0,y1,y2), paris.f90:2390-2411 (QUICK branch)
__device__ inline double inter(double x0, double x1, double x2, double x, double y0, double y1, double y2) {
    double xi = (x - x0) / (x1 - x0);
    double k = (x2 - x0) / (x1 - x0);
    double a = (y2 - k * k * y1 + (k * k - 1.0) * y0) / k / (1.0 - k);
    double b = (y2 - k * y1 + (k - 1.0) * y0) / k / (k - 1.0);
    return y0 + a * xi + b * (xi * xi);
}

// QUICK value of a component at its own cell centre ii along its axis
// (work(:,:,:,d) of the component's own direction): phi at n, stride st
__device__ inline double quick_same(const double* __restrict__ phi, long n, long st, const Ax& A, int ii, int g) {
    double pm1 = phi[n - st], p0 = phi[n];
    if (pm1 + p0 > 0.0)
        return inter(A.h[ii - 1 + g], A.h[ii + g], A.h[ii - 2 + g], A.c[ii + g], pm1, p0, phi[n - 2 * st]);
    return inter(A.h[ii + g], A.h[ii - 1 + g], A.h[ii + 1 + g], A.c[ii + g], p0, pm1, phi[n + st]);
}

// QUICK value of a component on the face jj+1/2 of another axis, upwinded
// by vel(n) + vel(n + sc)
__device__ inline double quick_cross(const double* __restrict__ phi, const double* __restrict__ vel, long n, long st,
                                     long sc, const Ax& A, int jj, int g) {
    if (vel[n] + vel[n + sc] > 0.0)
        return inter(A.c[jj + g], A.c[jj + 1 + g], A.c[jj - 1 + g], A.h[jj + g], phi[n], phi[n + st], phi[n - st]);
    return inter(A.c[jj + 1 + g], A.c[jj + g], A.c[jj + 2 + g], A.h[jj + g], phi[n + st], phi[n], phi[n + 2 * st]);
}

__device__ inline long stride(const Layout& L, int a) { return a == 0 ? 1 : (a == 1 ? L.pitch : L.plane); }

// momentumConvectionQUICK: du, dv, dw assigned on the faces project_velocity
// updates (is..ieu etc.)
__global__ void k_conv_quick(Vel V, double* __restrict__ du, double* __restrict__ dv, double* __restrict__ dw,
                             const Layout L, const Bnd B, const Geo G) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const long n = lidx(L, i, j, k), sx = 1, sy = L.pitch, sz = L.plane;
    const double *u = V.u, *v = V.v, *w = V.w;
    const Ax &X = G.a[0], &Y = G.a[1], &Z = G.a[2];
    if (i < L.n[0] - 1 || B.per[0]) {
        double a = quick_same(u, n + sx, sx, X, i + 1, g), b = quick_same(u, n, sx, X, i, g);
        double w2 = quick_cross(u, v, n, sy, sx, Y, j, g), w2m = quick_cross(u, v, n - sy, sy, sx, Y, j - 1, g);
        double w3 = quick_cross(u, w, n, sz, sx, Z, k, g), w3m = quick_cross(u, w, n - sz, sz, sx, Z, k - 1, g);
        du[n] = -(a * a - b * b) / X.dh[i + g]
            - 0.5 * ((v[n] + v[n + sx]) * w2 - (v[n - sy] + v[n + sx - sy]) * w2m) / Y.d[j + g]
            - 0.5 * ((w[n] + w[n + sx]) * w3 - (w[n - sz] + w[n + sx - sz]) * w3m) / Z.d[k + g];
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        double a = quick_same(v, n + sy, sy, Y, j + 1, g), b = quick_same(v, n, sy, Y, j, g);
        double w1 = quick_cross(v, u, n, sx, sy, X, i, g), w1m = quick_cross(v, u, n - sx, sx, sy, X, i - 1, g);
        double w3 = quick_cross(v, w, n, sz, sy, Z, k, g), w3m = quick_cross(v, w, n - sz, sz, sy, Z, k - 1, g);
        dv[n] = -0.5 * ((u[n] + u[n + sy]) * w1 - (u[n - sx] + u[n - sx + sy]) * w1m) / X.d[i + g]
            - (a * a - b * b) / Y.dh[j + g]
            - 0.5 * ((w[n] + w[n + sy]) * w3 - (w[n - sz] + w[n + sy - sz]) * w3m) / Z.d[k + g];
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        double a = quick_same(w, n + sz, sz, Z, k + 1, g), b = quick_same(w, n, sz, Z, k, g);
        double w1 = quick_cross(w, u, n, sx, sz, X, i, g), w1m = quick_cross(w, u, n - sx, sx, sz, X, i - 1, g);
        double w2 = quick_cross(w, v, n, sy, sz, Y, j, g), w2m = quick_cross(w, v, n - sy, sy, sz, Y, j - 1, g);
        dw[n] = -0.5 * ((u[n] + u[n + sz]) * w1 - (u[n - sx] + u[n - sx + sz]) * w1m) / X.d[i + g]
            - 0.5 * ((v[n] + v[n + sz]) * w2 - (v[n - sy] + v[n - sy + sz]) * w2m) / Y.d[j + g]
            - (a * a - b * b) / Z.dh[k + g];
    }
}

// minabs / maxabs (paris.f90:3450-3475) and slope_lim (modules.f90:177-197)
__device__ inline double minabs(double a, double b) { return fabs(a) < fabs(b) ? a : b; }
__device__ inline double maxabs(double a, double b) { return fabs(a) > fabs(b) ? a : b; }
__device__ inline double slope_lim(double v1, double v2, double v3, int scheme) {
    if (scheme == PARIS_CONV_SUPERBEE) {
        double a1 = minabs(v3 - v2, 2.0 * (v2 - v1));
        double a2 = minabs(2.0 * (v3 - v2), v2 - v1);
        return maxabs(a1, a2);
    } else if (scheme == PARIS_CONV_ENO) {
        return minabs(v3 - v2, v2 - v1);
    } else if (scheme == PARIS_CONV_WENO) {
        double d1 = v2 - v1, d2 = v3 - v2;
        double a1 = 1.0 / (d1 * d1 + 1.e-16);
        double a2 = 1.0 / (d2 * d2 + 1.e-16);
        double a = a1 + a2;
        return (a1 * (v2 - v1) + a2 * (v3 - v2)) / a;
    }
    return 0.0;
}

// work(p, a) of momentumConvection_onedim for the component phi of
// direction d (stride so = stride of d): the face value on axis a (stride
// sa, transport velocity vel) at cell n; oa = 1 when a == d
__device__ inline double eno_face(const double* __restrict__ phi, const double* __restrict__ vel, long n, long sa,
                                  long so, int oa, int scheme) {
    const long b = n - (oa ? sa : 0);              // p - oa e_a
    const long other = so - (oa ? sa : 0);         // o - oa e_a
    if (vel[b] + vel[n + other] > 0.0)
        return phi[b] + 0.5 * slope_lim(phi[b - sa], phi[b], phi[b + sa], scheme);
    return phi[b + sa] - 0.5 * slope_lim(phi[b], phi[b + sa], phi[b + 2 * sa], scheme);
}

// dphi = convection of component d (0..2) by the one-dimensional scheme
__device__ inline double eno_dphi(const Vel& V, const double* __restrict__ phi, long n, const Layout& L, int d,
                                  const Geo& G, int i, int j, int k, int scheme) {
    const int g = L.ng;
    const long s[3] = {1, L.pitch, L.plane};
    const long so = s[d];
    const double* vel[3] = {V.u, V.v, V.w};
    const int ix[3] = {i, j, k};
    double r = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const long sa = s[a];
        const int oa = a == d;
        const double* ve = vel[a];
        // (vel(p) + vel(p+o)) work(p + oa e_a) - (vel(p - e_a + oa e_a) + vel(p - e_a + o - oa e_a)) work(p - e_a + oa e_a)
        const long p1 = n + (oa ? sa : 0), p0 = n - sa + (oa ? sa : 0);
        double t = (ve[n] + ve[n + so]) * eno_face(phi, ve, p1, sa, so, oa, scheme) -
                   (ve[p0] + ve[n - sa + so - (oa ? sa : 0)]) * eno_face(phi, ve, p0, sa, so, oa, scheme);
        double term = 0.5 * t / G.a[a].d[ix[a] + g];
        r = a == 0 ? -term : r - term;
    }
    return r;
}

__global__ void k_conv_onedim(Vel V, double* __restrict__ du, double* __restrict__ dv, double* __restrict__ dw,
                              const Layout L, const Bnd B, const Geo G, int scheme) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const long n = lidx(L, i, j, k);
    if (i < L.n[0] - 1 || B.per[0]) du[n] = eno_dphi(V, V.u, n, L, 0, G, i, j, k, scheme);
    if (j < L.n[1] - 1 || B.per[1]) dv[n] = eno_dphi(V, V.v, n, L, 1, G, i, j, k, scheme);
    if (k < L.n[2] - 1 || B.per[2]) dw[n] = eno_dphi(V, V.w, n, L, 2, G, i, j, k, scheme);
}

}  // namespace

namespace {

// explicitMomDiff, paris.f90:2757-2808 (adds to du, dv, dw)
__global__ void k_mom_diff(Vel V, const double* __restrict__ rho, const double* __restrict__ mu,
                           double* __restrict__ du, double* __restrict__ dv, double* __restrict__ dw, const Layout L,
                           const Bnd B, const Geo G) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const long n = lidx(L, i, j, k), sx = 1, sy = L.pitch, sz = L.plane;
    const double *u = V.u, *v = V.v, *w = V.w;
    const double *dx = G.a[0].d, *dxh = G.a[0].dh, *dy = G.a[1].d, *dyh = G.a[1].dh, *dz = G.a[2].d,
                 *dzh = G.a[2].dh;
    const int I = i + g, J = j + g, K = k + g;   // metric index
#define M(o) mu[n + (o)]
#define U(o) u[n + (o)]
#define VV(o) v[n + (o)]
#define W(o) w[n + (o)]
    if (i < L.n[0] - 1 || B.per[0]) {
        du[n] = du[n] + (
            (1. / dxh[I]) * 2. * (M(sx) * (1. / dx[I + 1]) * (U(sx) - U(0)) - M(0) * (1. / dx[I]) * (U(0) - U(-sx)))
            + (1. / dy[J]) * (0.25 * (M(0) + M(sx) + M(sx + sy) + M(sy)) *
                                  ((1. / dyh[J]) * (U(sy) - U(0)) + (1. / dxh[I]) * (VV(sx) - VV(0))) -
                              0.25 * (M(0) + M(sx) + M(sx - sy) + M(-sy)) *
                                  ((1. / dyh[J - 1]) * (U(0) - U(-sy)) + (1. / dxh[I]) * (VV(sx - sy) - VV(-sy))))
            + (1. / dz[K]) * (0.25 * (M(0) + M(sx) + M(sx + sz) + M(sz)) *
                                  ((1. / dzh[K]) * (U(sz) - U(0)) + (1. / dxh[I]) * (W(sx) - W(0))) -
                              0.25 * (M(0) + M(sx) + M(sx - sz) + M(-sz)) *
                                  ((1. / dzh[K - 1]) * (U(0) - U(-sz)) + (1. / dxh[I]) * (W(sx - sz) - W(-sz))))
            ) / (0.5 * (rho[n + sx] + rho[n]));
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        dv[n] = dv[n] + (
            (1. / dx[I]) * (0.25 * (M(0) + M(sx) + M(sx + sy) + M(sy)) *
                                ((1. / dyh[J]) * (U(sy) - U(0)) + (1. / dxh[I]) * (VV(sx) - VV(0))) -
                            0.25 * (M(0) + M(sy) + M(sy - sx) + M(-sx)) *
                                ((1. / dyh[J]) * (U(sy - sx) - U(-sx)) + (1. / dxh[I - 1]) * (VV(0) - VV(-sx))))
            + (1. / dyh[J]) * 2. * (M(sy) * (1. / dy[J + 1]) * (VV(sy) - VV(0)) - M(0) * (1. / dy[J]) * (VV(0) - VV(-sy)))
            + (1. / dz[K]) * (0.25 * (M(0) + M(sy) + M(sy + sz) + M(sz)) *
                                  ((1. / dzh[K]) * (VV(sz) - VV(0)) + (1. / dyh[J]) * (W(sy) - W(0))) -
                              0.25 * (M(0) + M(sy) + M(sy - sz) + M(-sz)) *
                                  ((1. / dzh[K - 1]) * (VV(0) - VV(-sz)) + (1. / dyh[J]) * (W(sy - sz) - W(-sz))))
            ) / (0.5 * (rho[n + sy] + rho[n]));
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        dw[n] = dw[n] + (
            (1. / dx[I]) * (0.25 * (M(0) + M(sx) + M(sx + sz) + M(sz)) *
                                ((1. / dzh[K]) * (U(sz) - U(0)) + (1. / dxh[I]) * (W(sx) - W(0))) -
                            0.25 * (M(0) + M(-sx) + M(-sx + sz) + M(sz)) *
                                ((1. / dzh[K]) * (U(-sx + sz) - U(-sx)) + (1. / dxh[I - 1]) * (W(0) - W(-sx))))
            + (1. / dy[J]) * (0.25 * (M(0) + M(sy) + M(sy + sz) + M(sz)) *
                                  ((1. / dzh[K]) * (VV(sz) - VV(0)) + (1. / dyh[J]) * (W(sy) - W(0))) -
                              0.25 * (M(0) + M(-sy) + M(-sy + sz) + M(sz)) *
                                  ((1. / dzh[K]) * (VV(-sy + sz) - VV(-sy)) + (1. / dyh[J - 1]) * (W(0) - W(-sy))))
            + (1. / dzh[K]) * 2. * (M(sz) * (1. / dz[K + 1]) * (W(sz) - W(0)) - M(0) * (1. / dz[K]) * (W(0) - W(-sz)))
            ) / (0.5 * (rho[n + sz] + rho[n]));
    }
#undef M
#undef U
#undef VV
#undef W
}

// volumeForce, paris.f90:2813-2860, with the front-tracking force zero
__global__ void k_volume_force(const double* __restrict__ rho, double* __restrict__ du, double* __restrict__ dv,
                               double* __restrict__ dw, const Layout L, const Bnd B, double dpdx, double dpdy,
                               double dpdz, double rro, double gx, double gy, double gz) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const long n = lidx(L, i, j, k);
    if (i < L.n[0] - 1 || B.per[0]) {
        double fx = 0.0 - dpdx + (0.5 * (rho[n + 1] + rho[n]) - rro) * gx;
        du[n] = du[n] + fx / (0.5 * (rho[n + 1] + rho[n]));
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        double fy = 0.0 - dpdy + (0.5 * (rho[n + L.pitch] + rho[n]) - rro) * gy;
        dv[n] = dv[n] + fy / (0.5 * (rho[n + L.pitch] + rho[n]));
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        double fz = 0.0 - dpdz + (0.5 * (rho[n + L.plane] + rho[n]) - rro) * gz;
        dw[n] = dw[n] + fz / (0.5 * (rho[n + L.plane] + rho[n]));
    }
}

// u = u + dt*du over the whole arrays, ghosts included
__global__ void k_advance(double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                          const double* __restrict__ du, const double* __restrict__ dv,
                          const double* __restrict__ dw, double dt, long total) {
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        u[t] = u[t] + dt * du[t];
        v[t] = v[t] + dt * dv[t];
        w[t] = w[t] + dt * dw[t];
    }
}

// SetVelocityBC for no-slip / moving walls, one direction at a time in the
// reference's order (x, then y, then z); each thread owns one line of the
// ghosted plane normal to that direction.  WV(f,c) = wv[(f-1) + 6 (c-1)].
struct WallV {
    double v[18];
};
__global__ void k_wall_bc(double* __restrict__ u, double* __restrict__ v, double* __restrict__ w, const Layout L,
                          int dir, int lo, int hi, WallV WV) {
    const int g = L.ng;
    const int ta = dir == 0 ? 1 : 0, tb = dir == 2 ? 1 : 2;   // the two transverse axes
    const int na = L.n[ta] + 2 * g, nb = L.n[tb] + 2 * g;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= na * nb) return;
    int ia = p % na - g, ib = p / na - g;
    int c[3];
    c[ta] = ia;
    c[tb] = ib;
    const long s = dir == 0 ? 1 : (dir == 1 ? L.pitch : L.plane);
    // normal component, and the two tangential ones in the reference's order
    double* nrm = dir == 0 ? u : (dir == 1 ? v : w);
    double* t1 = dir == 0 ? v : u;
    double* t2 = dir == 2 ? v : w;
    const int c1 = dir == 0 ? 2 : 1, c2 = dir == 2 ? 2 : 3;   // WallVel component of t1, t2
    auto WVf = [&](int f, int comp) { return WV.v[(f - 1) + 6 * (comp - 1)]; };
    const int nd = L.n[dir];
    if (lo) {   // face 2*dir+1: nrm(is-1) = 0, nrm(is-2) = -nrm(is), t = 2 WV - t(is)
        c[dir] = 0;
        long n0 = lidx(L, c[0], c[1], c[2]);
        const int f = 2 * dir + 1;
        nrm[n0 - s] = 0.0;
        nrm[n0 - 2 * s] = -nrm[n0];
        t1[n0 - s] = 2 * WVf(f, c1) - t1[n0];
        t2[n0 - s] = 2 * WVf(f, c2) - t2[n0];
    }
    if (hi) {   // face 2*dir+2: nrm(ie) = 0, nrm(ie+1) = -nrm(ie-1), t(ie+1) = 2 WV - t(ie)
        c[dir] = nd - 1;
        long ne = lidx(L, c[0], c[1], c[2]);
        const int f = 2 * dir + 2;
        nrm[ne] = 0.0;
        nrm[ne + s] = -nrm[ne - s];
        t1[ne + s] = 2 * WVf(f, c1) - t1[ne];
        t2[ne + s] = 2 * WVf(f, c2) - t2[ne];
    }
}

inline dim3 cblock() { return dim3(128, 2, 1); }
inline dim3 cgrid(const Layout& L) { return dim3(div_up(L.n[0], 128), div_up(L.n[1], 2), L.n[2]); }

Geo geo(const paris_ctx* c) {
    return Geo{{Ax{c->xc, c->xh, c->dx, c->dxh}, Ax{c->yc, c->yh, c->dy, c->dyh}, Ax{c->zc, c->zh, c->dz, c->dzh}}};
}
Vel vel(const paris_ctx* c) { return Vel{c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W]}; }

int need(paris_ctx* c, std::initializer_list<int> fields) {
    for (int f : fields) PARIS_CHECK(ctx_alloc_field(c, f));
    return PARIS_OK;
}

}  // namespace

extern "C" int paris_momentum_convection(paris_handle_t c, int32_t scheme) {
    if (!c) return PARIS_BAD_ARGS;
    if (scheme < PARIS_CONV_QUICK || scheme > PARIS_CONV_WENO) {
        ctx_set_error(c, "momentumConvection: unknown scheme %d", scheme);
        return PARIS_BAD_ARGS;
    }
    cudaSetDevice(c->dev);
    PARIS_CHECK(need(c, {PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}));
    if (scheme == PARIS_CONV_QUICK)
        PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_quick, cgrid(c->L), cblock(), 0, vel(c), c->fld[PARIS_FIELD_DU],
                       c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, geo(c));
    else
        PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_onedim, cgrid(c->L), cblock(), 0, vel(c),
                       c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, geo(c),
                       scheme);
    return PARIS_OK;
}

extern "C" int paris_explicit_mom_diff(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(need(c, {PARIS_FIELD_MU, PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}));
    PARIS_LAUNCH_N(c, "mom_diffusion", c->N, k_mom_diff, cgrid(c->L), cblock(), 0, vel(c), c->fld[PARIS_FIELD_RHO],
                   c->fld[PARIS_FIELD_MU], c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L,
                   c->bnd, geo(c));
    return PARIS_OK;
}

extern "C" int paris_volume_force(paris_handle_t c, double dpdx, double dpdy, double dpdz, int32_t buoyancy, double gx,
                                  double gy, double gz, double rho_ave) {
    if (!c) return PARIS_BAD_ARGS;
    double rro;
    if (buoyancy == 0) rro = 0.0;
    else if (buoyancy == 1) rro = c->d.rho1;
    else if (buoyancy == 2) rro = c->d.rho2;
    else if (buoyancy == 3) rro = rho_ave;
    else {
        ctx_set_error(c, "volumeForce: invalid buoyancy option %d", buoyancy);
        return PARIS_BAD_ARGS;
    }
    cudaSetDevice(c->dev);
    PARIS_CHECK(need(c, {PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}));
    PARIS_LAUNCH_N(c, "volume_force", c->N, k_volume_force, cgrid(c->L), cblock(), 0, c->fld[PARIS_FIELD_RHO],
                   c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, dpdx, dpdy,
                   dpdz, rro, gx, gy, gz);
    return PARIS_OK;
}

extern "C" int paris_advance_velocity(paris_handle_t c, double dt) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(need(c, {PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}));
    const long T = c->L.total;
    PARIS_LAUNCH_N(c, "advance_velocity", c->N, k_advance, (unsigned)div_up(T, 256L * 4), 256, 0,
                   c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W], c->fld[PARIS_FIELD_DU],
                   c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], dt, T);
    return PARIS_OK;
}

extern "C" int paris_set_velocity_bc(paris_handle_t c, const double* wall_vel) {
    if (!c) return PARIS_BAD_ARGS;
    for (int f = 0; f < 6; f++)
        if (c->d.bdry_cond[f] != PARIS_BC_WALL && c->d.bdry_cond[f] != PARIS_BC_PERIODIC) {
            ctx_set_error(c, "SetVelocityBC: only walls (0) and periodic (1) boundaries are supported");
            return PARIS_BAD_ARGS;
        }
    cudaSetDevice(c->dev);
    WallV WV{};
    if (wall_vel)
        for (int q = 0; q < 18; q++) WV.v[q] = wall_vel[q];
    for (int dir = 0; dir < 3; dir++) {
        const int lo = c->d.bdry_cond[dir] == PARIS_BC_WALL, hi = c->d.bdry_cond[dir + 3] == PARIS_BC_WALL;
        if (!lo && !hi) continue;
        const int ta = dir == 0 ? 1 : 0, tb = dir == 2 ? 1 : 2;
        const long lines = (long)(c->L.n[ta] + 2 * c->L.ng) * (c->L.n[tb] + 2 * c->L.ng);
        PARIS_LAUNCH_N(c, "velocity_bc", lines, k_wall_bc, (unsigned)div_up(lines, 256L), 256, 0,
                       c->fld[PARIS_FIELD_U], c->fld[PARIS_FIELD_V], c->fld[PARIS_FIELD_W], c->L, dir, lo, hi, WV);
    }
    // do_ghost_vector: the periodic images
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_U]));
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_V]));
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[PARIS_FIELD_W]));
    return PARIS_OK;
}
