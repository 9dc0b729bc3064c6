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
#include <cmath>

#include "ctx.cuh"
#include "limiter.cuh"

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

// The coordinate part of inter() for one face: xi and k from x0, x1, x2, x,
// computed once per index on the host with the same IEEE operations (so the
// values are those inter() forms), plus the reciprocals of k, 1 - k, k - 1.
// On a uniform grid with a power-of-two cell count k = -1, so the divisions
// of inter() by k, 1 - k and k - 1 are by powers of two: multiplying by the
// exact reciprocal then rounds to the same double as dividing, and the
// kernel takes that form (R = true) when every reciprocal it uses is exact.
struct QuickCoef {
    double xi, k, rk, r1k, rkm1;
};
// Per axis, index t = ii + ng: Q[4t + 0] own axis, vel > 0; 4t + 1 own
// axis, otherwise; 4t + 2 cross axis, vel > 0; 4t + 3 cross axis, otherwise.
// rd = 1./d, rdh = 1./dh (the metric reciprocals of explicitMomDiff).
struct MomTab {
    const QuickCoef* q[3];
    const double* rd[3];
    const double* rdh[3];
};

// inter(x0,x1,x2,x,y0,y1,y2), paris.f90:2390-2411 (QUICK branch), with the
// coordinate part from the table
template <bool R>
__device__ inline double inter_q(const QuickCoef* __restrict__ c, double y0, double y1, double y2) {
    const double k = c->k, xi = c->xi;
    double a, b;
    if (R) {
        a = ((y2 - k * k * y1 + (k * k - 1.0) * y0) * c->rk) * c->r1k;
        b = ((y2 - k * y1 + (k - 1.0) * y0) * c->rk) * c->rkm1;
    } else {
        a = (y2 - k * k * y1 + (k * k - 1.0) * y0) / k / (1.0 - k);
        b = (y2 - k * y1 + (k - 1.0) * y0) / k / (k - 1.0);
    }
    return y0 + a * xi + b * (xi * xi);
}

// QUICK value of a component at its own cell centre ii along its axis
// (work(:,:,:,d) of the component's own direction): phi at n, stride st
// Both candidates of the upwind point are loaded before the upwind test, so
// the four loads of a face value are independent (one memory round trip
// instead of two); the arithmetic is unchanged.
template <bool R>
__device__ inline double quick_same(const double* __restrict__ phi, long n, long st, const QuickCoef* __restrict__ Q,
                                    int t) {
    const double pm2 = phi[n - 2 * st], pm1 = phi[n - st], p0 = phi[n], pp1 = phi[n + st];
    const bool up = pm1 + p0 > 0.0;
    const double y2 = up ? pm2 : pp1;
    return inter_q<R>(Q + 4 * t + (up ? 0 : 1), up ? pm1 : p0, up ? p0 : pm1, y2);
}
// the same with the two coefficient sets of a uniform axis
__device__ inline QuickCoef pick(bool up, const QuickCoef& a, const QuickCoef& b) {
    return QuickCoef{up ? a.xi : b.xi, up ? a.k : b.k, up ? a.rk : b.rk, up ? a.r1k : b.r1k, up ? a.rkm1 : b.rkm1};
}
// inter_q<true> for the coefficients of every face of a uniform grid whose
// coordinates are exact (xi = 1/2, k = -1, so k*k = 1, k*k - 1 = 0, k - 1 = -2,
// 1/k = -1, 1/(1-k) = 1/2, 1/(k-1) = -1/2): the same IEEE operations with
// those constants, the exact products by -1 folded into the scalings
// ((x * -1) * 1/2 and x * -1/2 round alike), so the same double as inter_q
__device__ inline double inter_canon(double y0, double y1, double y2) {
    const double a = ((y2 - y1) + 0.0 * y0) * -0.5;
    const double b = ((y2 + y1) + -2.0 * y0) * 0.5;
    return (y0 + a * 0.5) + b * 0.25;
}
template <bool C>
__device__ inline double inter_u(const QuickCoef& c, double y0, double y1, double y2) {
    return C ? inter_canon(y0, y1, y2) : inter_q<true>(&c, y0, y1, y2);
}
template <bool C>
__device__ inline double quick_same_u(const double* __restrict__ phi, long n, long st, const QuickCoef& cu,
                                      const QuickCoef& cd) {
    const double pm2 = phi[n - 2 * st], pm1 = phi[n - st], p0 = phi[n], pp1 = phi[n + st];
    const bool up = pm1 + p0 > 0.0;
    const QuickCoef c = C ? cu : pick(up, cu, cd);
    return inter_u<C>(c, up ? pm1 : p0, up ? p0 : pm1, up ? pm2 : pp1);
}

// QUICK value of a component on the face jj+1/2 of another axis, upwinded
// by vel(n) + vel(n + sc)
template <bool R>
__device__ inline double quick_cross(const double* __restrict__ phi, const double* __restrict__ vel, long n, long st,
                                     long sc, const QuickCoef* __restrict__ Q, int t) {
    const double v0 = vel[n], v1 = vel[n + sc];
    const double am = phi[n - st], a = phi[n], b = phi[n + st], bp = phi[n + 2 * st];
    const bool up = v0 + v1 > 0.0;
    return inter_q<R>(Q + 4 * t + (up ? 2 : 3), up ? a : b, up ? b : a, up ? am : bp);
}
template <bool C>
__device__ inline double quick_cross_u(const double* __restrict__ phi, const double* __restrict__ vel, long n, long st,
                                       long sc, const QuickCoef& cu, const QuickCoef& cd) {
    const double v0 = vel[n], v1 = vel[n + sc];
    const double am = phi[n - st], a = phi[n], b = phi[n + st], bp = phi[n + 2 * st];
    const bool up = v0 + v1 > 0.0;
    const QuickCoef c = C ? cu : pick(up, cu, cd);
    return inter_u<C>(c, up ? a : b, up ? b : a, up ? am : bp);
}

// x / den, or x * (1/den) where that reciprocal is exact (same double)
template <bool R>
__device__ inline double over(double x, double den, double rden) {
    return R ? x * rden : x / den;
}

// The coefficients of a uniform grid: every index carries the same four
// coefficient sets and metric reciprocals per axis (checked bit for bit on
// the host), passed by value so the kernel loads no table.
struct QuickUniform {
    QuickCoef q[3][4];
    double d[3], dh[3], rd[3], rdh[3];
};

// momentumConvectionQUICK: du, dv, dw assigned on the faces project_velocity
// updates (is..ieu etc.)
template <bool R>
__global__ void __launch_bounds__(256) k_conv_quick(Vel V, double* __restrict__ du, double* __restrict__ dv,
                                                    double* __restrict__ dw, const Layout L, const Bnd B, const Geo G,
                                                    const MomTab T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const long n = lidx(L, i, j, k), sx = 1, sy = L.pitch, sz = L.plane;
    const double *u = V.u, *v = V.v, *w = V.w;
    const QuickCoef *QX = T.q[0], *QY = T.q[1], *QZ = T.q[2];
    const int I = i + g, J = j + g, K = k + g;
    if (i < L.n[0] - 1 || B.per[0]) {
        double a = quick_same<R>(u, n + sx, sx, QX, I + 1), b = quick_same<R>(u, n, sx, QX, I);
        double w2 = quick_cross<R>(u, v, n, sy, sx, QY, J), w2m = quick_cross<R>(u, v, n - sy, sy, sx, QY, J - 1);
        double w3 = quick_cross<R>(u, w, n, sz, sx, QZ, K), w3m = quick_cross<R>(u, w, n - sz, sz, sx, QZ, K - 1);
        du[n] = over<R>(-(a * a - b * b), G.a[0].dh[I], T.rdh[0][I])
            - over<R>(0.5 * ((v[n] + v[n + sx]) * w2 - (v[n - sy] + v[n + sx - sy]) * w2m), G.a[1].d[J], T.rd[1][J])
            - over<R>(0.5 * ((w[n] + w[n + sx]) * w3 - (w[n - sz] + w[n + sx - sz]) * w3m), G.a[2].d[K], T.rd[2][K]);
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        double a = quick_same<R>(v, n + sy, sy, QY, J + 1), b = quick_same<R>(v, n, sy, QY, J);
        double w1 = quick_cross<R>(v, u, n, sx, sy, QX, I), w1m = quick_cross<R>(v, u, n - sx, sx, sy, QX, I - 1);
        double w3 = quick_cross<R>(v, w, n, sz, sy, QZ, K), w3m = quick_cross<R>(v, w, n - sz, sz, sy, QZ, K - 1);
        dv[n] = over<R>(-0.5 * ((u[n] + u[n + sy]) * w1 - (u[n - sx] + u[n - sx + sy]) * w1m), G.a[0].d[I], T.rd[0][I])
            - over<R>(a * a - b * b, G.a[1].dh[J], T.rdh[1][J])
            - over<R>(0.5 * ((w[n] + w[n + sy]) * w3 - (w[n - sz] + w[n + sy - sz]) * w3m), G.a[2].d[K], T.rd[2][K]);
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        double a = quick_same<R>(w, n + sz, sz, QZ, K + 1), b = quick_same<R>(w, n, sz, QZ, K);
        double w1 = quick_cross<R>(w, u, n, sx, sz, QX, I), w1m = quick_cross<R>(w, u, n - sx, sx, sz, QX, I - 1);
        double w2 = quick_cross<R>(w, v, n, sy, sz, QY, J), w2m = quick_cross<R>(w, v, n - sy, sy, sz, QY, J - 1);
        dw[n] = over<R>(-0.5 * ((u[n] + u[n + sz]) * w1 - (u[n - sx] + u[n - sx + sz]) * w1m), G.a[0].d[I], T.rd[0][I])
            - over<R>(0.5 * ((v[n] + v[n + sz]) * w2 - (v[n - sy] + v[n - sy + sz]) * w2m), G.a[1].d[J], T.rd[1][J])
            - over<R>(a * a - b * b, G.a[2].dh[K], T.rdh[2][K]);
    }
}

// momentumConvectionQUICK on a uniform grid with exact reciprocals; C: every
// coefficient set is the exact-coordinate one (inter_canon)
template <bool C>
__global__ void __launch_bounds__(256) k_conv_quick_uniform(Vel V, double* __restrict__ du, double* __restrict__ dv,
                                                            double* __restrict__ dw, const Layout L, const Bnd B,
                                                            const QuickUniform Q) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const long n = lidx(L, i, j, k), sx = 1, sy = L.pitch, sz = L.plane;
    const double *u = V.u, *v = V.v, *w = V.w;
    if (i < L.n[0] - 1 || B.per[0]) {
        double a = quick_same_u<C>(u, n + sx, sx, Q.q[0][0], Q.q[0][1]), b = quick_same_u<C>(u, n, sx, Q.q[0][0], Q.q[0][1]);
        double w2 = quick_cross_u<C>(u, v, n, sy, sx, Q.q[1][2], Q.q[1][3]);
        double w2m = quick_cross_u<C>(u, v, n - sy, sy, sx, Q.q[1][2], Q.q[1][3]);
        double w3 = quick_cross_u<C>(u, w, n, sz, sx, Q.q[2][2], Q.q[2][3]);
        double w3m = quick_cross_u<C>(u, w, n - sz, sz, sx, Q.q[2][2], Q.q[2][3]);
        du[n] = -(a * a - b * b) * Q.rdh[0]
            - (0.5 * ((v[n] + v[n + sx]) * w2 - (v[n - sy] + v[n + sx - sy]) * w2m)) * Q.rd[1]
            - (0.5 * ((w[n] + w[n + sx]) * w3 - (w[n - sz] + w[n + sx - sz]) * w3m)) * Q.rd[2];
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        double a = quick_same_u<C>(v, n + sy, sy, Q.q[1][0], Q.q[1][1]), b = quick_same_u<C>(v, n, sy, Q.q[1][0], Q.q[1][1]);
        double w1 = quick_cross_u<C>(v, u, n, sx, sy, Q.q[0][2], Q.q[0][3]);
        double w1m = quick_cross_u<C>(v, u, n - sx, sx, sy, Q.q[0][2], Q.q[0][3]);
        double w3 = quick_cross_u<C>(v, w, n, sz, sy, Q.q[2][2], Q.q[2][3]);
        double w3m = quick_cross_u<C>(v, w, n - sz, sz, sy, Q.q[2][2], Q.q[2][3]);
        dv[n] = (-0.5 * ((u[n] + u[n + sy]) * w1 - (u[n - sx] + u[n - sx + sy]) * w1m)) * Q.rd[0]
            - (a * a - b * b) * Q.rdh[1]
            - (0.5 * ((w[n] + w[n + sy]) * w3 - (w[n - sz] + w[n + sy - sz]) * w3m)) * Q.rd[2];
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        double a = quick_same_u<C>(w, n + sz, sz, Q.q[2][0], Q.q[2][1]), b = quick_same_u<C>(w, n, sz, Q.q[2][0], Q.q[2][1]);
        double w1 = quick_cross_u<C>(w, u, n, sx, sz, Q.q[0][2], Q.q[0][3]);
        double w1m = quick_cross_u<C>(w, u, n - sx, sx, sz, Q.q[0][2], Q.q[0][3]);
        double w2 = quick_cross_u<C>(w, v, n, sy, sz, Q.q[1][2], Q.q[1][3]);
        double w2m = quick_cross_u<C>(w, v, n - sy, sy, sz, Q.q[1][2], Q.q[1][3]);
        dw[n] = (-0.5 * ((u[n] + u[n + sz]) * w1 - (u[n - sx] + u[n - sx + sz]) * w1m)) * Q.rd[0]
            - (0.5 * ((v[n] + v[n + sz]) * w2 - (v[n - sy] + v[n - sy + sz]) * w2m)) * Q.rd[1]
            - (a * a - b * b) * Q.rdh[2];
    }
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
template <bool UNI>
__global__ void __launch_bounds__(256) k_mom_diff(Vel V, const double* __restrict__ rho, const double* __restrict__ mu,
                                                  double* __restrict__ du, double* __restrict__ dv,
                                                  double* __restrict__ dw, const Layout L, const Bnd B, const MomTab T,
                                                  const QuickUniform Q) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) return;
    const int g = L.ng;
    const long n = lidx(L, i, j, k), sx = 1, sy = L.pitch, sz = L.plane;
    const double *u = V.u, *v = V.v, *w = V.w;
    // 1./dx(i) etc. from the table (the same IEEE divisions, done once per
    // index), or on a uniform grid the one value every index holds
    const double *rdx = T.rd[0], *rdxh = T.rdh[0], *rdy = T.rd[1], *rdyh = T.rdh[1], *rdz = T.rd[2],
                 *rdzh = T.rdh[2];
#define RD(p, a, t) (UNI ? Q.rd[a] : p[t])
#define RDH(p, a, t) (UNI ? Q.rdh[a] : p[t])
    const int I = i + g, J = j + g, K = k + g;   // metric index
#define M(o) mu[n + (o)]
#define U(o) u[n + (o)]
#define VV(o) v[n + (o)]
#define W(o) w[n + (o)]
    if (i < L.n[0] - 1 || B.per[0]) {
        du[n] = du[n] + (
            RDH(rdxh, 0, I) * 2. * (M(sx) * RD(rdx, 0, I + 1) * (U(sx) - U(0)) - M(0) * RD(rdx, 0, I) * (U(0) - U(-sx)))
            + RD(rdy, 1, J) * (0.25 * (M(0) + M(sx) + M(sx + sy) + M(sy)) *
                                  (RDH(rdyh, 1, J) * (U(sy) - U(0)) + RDH(rdxh, 0, I) * (VV(sx) - VV(0))) -
                              0.25 * (M(0) + M(sx) + M(sx - sy) + M(-sy)) *
                                  (RDH(rdyh, 1, J - 1) * (U(0) - U(-sy)) + RDH(rdxh, 0, I) * (VV(sx - sy) - VV(-sy))))
            + RD(rdz, 2, K) * (0.25 * (M(0) + M(sx) + M(sx + sz) + M(sz)) *
                                  (RDH(rdzh, 2, K) * (U(sz) - U(0)) + RDH(rdxh, 0, I) * (W(sx) - W(0))) -
                              0.25 * (M(0) + M(sx) + M(sx - sz) + M(-sz)) *
                                  (RDH(rdzh, 2, K - 1) * (U(0) - U(-sz)) + RDH(rdxh, 0, I) * (W(sx - sz) - W(-sz))))
            ) / (0.5 * (rho[n + sx] + rho[n]));
    }
    if (j < L.n[1] - 1 || B.per[1]) {
        dv[n] = dv[n] + (
            RD(rdx, 0, I) * (0.25 * (M(0) + M(sx) + M(sx + sy) + M(sy)) *
                                (RDH(rdyh, 1, J) * (U(sy) - U(0)) + RDH(rdxh, 0, I) * (VV(sx) - VV(0))) -
                            0.25 * (M(0) + M(sy) + M(sy - sx) + M(-sx)) *
                                (RDH(rdyh, 1, J) * (U(sy - sx) - U(-sx)) + RDH(rdxh, 0, I - 1) * (VV(0) - VV(-sx))))
            + RDH(rdyh, 1, J) * 2. * (M(sy) * RD(rdy, 1, J + 1) * (VV(sy) - VV(0)) - M(0) * RD(rdy, 1, J) * (VV(0) - VV(-sy)))
            + RD(rdz, 2, K) * (0.25 * (M(0) + M(sy) + M(sy + sz) + M(sz)) *
                                  (RDH(rdzh, 2, K) * (VV(sz) - VV(0)) + RDH(rdyh, 1, J) * (W(sy) - W(0))) -
                              0.25 * (M(0) + M(sy) + M(sy - sz) + M(-sz)) *
                                  (RDH(rdzh, 2, K - 1) * (VV(0) - VV(-sz)) + RDH(rdyh, 1, J) * (W(sy - sz) - W(-sz))))
            ) / (0.5 * (rho[n + sy] + rho[n]));
    }
    if (k < L.n[2] - 1 || B.per[2]) {
        dw[n] = dw[n] + (
            RD(rdx, 0, I) * (0.25 * (M(0) + M(sx) + M(sx + sz) + M(sz)) *
                                (RDH(rdzh, 2, K) * (U(sz) - U(0)) + RDH(rdxh, 0, I) * (W(sx) - W(0))) -
                            0.25 * (M(0) + M(-sx) + M(-sx + sz) + M(sz)) *
                                (RDH(rdzh, 2, K) * (U(-sx + sz) - U(-sx)) + RDH(rdxh, 0, I - 1) * (W(0) - W(-sx))))
            + RD(rdy, 1, J) * (0.25 * (M(0) + M(sy) + M(sy + sz) + M(sz)) *
                                  (RDH(rdzh, 2, K) * (VV(sz) - VV(0)) + RDH(rdyh, 1, J) * (W(sy) - W(0))) -
                              0.25 * (M(0) + M(-sy) + M(-sy + sz) + M(sz)) *
                                  (RDH(rdzh, 2, K) * (VV(-sy + sz) - VV(-sy)) + RDH(rdyh, 1, J - 1) * (W(0) - W(-sy))))
            + RDH(rdzh, 2, K) * 2. * (M(sz) * RD(rdz, 2, K + 1) * (W(sz) - W(0)) - M(0) * RD(rdz, 2, K) * (W(0) - W(-sz)))
            ) / (0.5 * (rho[n + sz] + rho[n]));
    }
#undef RD
#undef RDH
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

bool pow2(double x) {
    int e;
    const double m = std::frexp(x, &e);
    return m == 0.5 || m == -0.5;
}

// The per-index tables of MomTab, built once per grid on the host from the
// host copies of the coordinates (the same doubles the device holds).
int mom_tables(paris_ctx* c, MomTab* T, bool* exact, QuickUniform* U = nullptr, bool* uniform = nullptr) {
    const int g = c->L.ng;
    const std::vector<double>* C[3] = {&c->h_x, &c->h_y, &c->h_z};
    const std::vector<double>* H[3] = {&c->h_xh, &c->h_yh, &c->h_zh};
    const std::vector<double>* D[3] = {&c->h_dx, &c->h_dy, &c->h_dz};
    const std::vector<double>* DH[3] = {&c->h_dxh, &c->h_dyh, &c->h_dzh};
    const int per = (int)(sizeof(QuickCoef) / sizeof(double));   // doubles per coefficient set
    long off[3], total = 0;
    for (int a = 0; a < 3; a++) {
        off[a] = total;
        total += (long)C[a]->size() * (4 * per + 2);
    }
    if (!c->mom_tab) {
        std::vector<double> tab(total, 0.0);
        bool ex = true;
        for (int a = 0; a < 3; a++) {
            const std::vector<double>&x = *C[a], &xh = *H[a], &d = *D[a], &dh = *DH[a];
            const int nt = (int)x.size(), n = c->L.n[a];
            QuickCoef* Q = reinterpret_cast<QuickCoef*>(tab.data() + off[a]);
            double* rd = tab.data() + off[a] + 4L * per * nt;
            double* rdh = rd + nt;
            // inter(x0,x1,x2,x): xi and k exactly as inter() forms them
            auto set = [&](QuickCoef& q, double x0, double x1, double x2, double xx, bool used) {
                q.xi = (xx - x0) / (x1 - x0);
                q.k = (x2 - x0) / (x1 - x0);
                const double omk = 1.0 - q.k, km1 = q.k - 1.0;
                q.rk = 1.0 / q.k;
                q.r1k = 1.0 / omk;
                q.rkm1 = 1.0 / km1;
                if (used) ex = ex && pow2(q.k) && pow2(omk) && pow2(km1);
            };
            for (int t = 0; t < nt; t++) {
                // own axis: ii = t - g in [0, n]; cross axis: jj = t - g in [-1, n-1]
                const bool own = t >= g && t <= n + g, cross = t >= g - 1 && t <= n + g - 1;
                if (t >= 2) set(Q[4 * t + 0], xh[t - 1], xh[t], xh[t - 2], x[t], own);
                if (t >= 1 && t + 1 < nt) set(Q[4 * t + 1], xh[t], xh[t - 1], xh[t + 1], x[t], own);
                if (t >= 1 && t + 1 < nt) set(Q[4 * t + 2], x[t], x[t + 1], x[t - 1], xh[t], cross);
                if (t + 2 < nt) set(Q[4 * t + 3], x[t + 1], x[t], x[t + 2], xh[t], cross);
                rd[t] = 1. / d[t];
                rdh[t] = 1. / dh[t];
                if (t >= g && t < n + g) ex = ex && pow2(d[t]) && pow2(dh[t]);
            }
        }
        PARIS_CUDA_TRY(c, cudaMalloc(&c->mom_tab, total * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMemcpy(c->mom_tab, tab.data(), total * sizeof(double), cudaMemcpyHostToDevice));
        c->mom_tab_exact = ex ? 1 : 0;
    }
    for (int a = 0; a < 3; a++) {
        const long nt = (long)C[a]->size();
        T->q[a] = reinterpret_cast<const QuickCoef*>(c->mom_tab + off[a]);
        T->rd[a] = c->mom_tab + off[a] + 4L * per * nt;
        T->rdh[a] = T->rd[a] + nt;
    }
    *exact = c->mom_tab_exact != 0;
    if (uniform) {
        // every index the kernel reads holds the same coefficients, bit for bit
        // (then rebuilt here from the host coordinates: same arithmetic)
        bool uni = *exact;
        for (int a = 0; a < 3 && uni; a++) {
            const std::vector<double>&x = *C[a], &xh = *H[a], &d = *D[a], &dh = *DH[a];
            const int n = c->L.n[a];
            auto coef = [&](int v, int t) {
                QuickCoef q;
                double x0, x1, x2, xx;
                if (v == 0) { x0 = xh[t - 1]; x1 = xh[t]; x2 = xh[t - 2]; xx = x[t]; }
                else if (v == 1) { x0 = xh[t]; x1 = xh[t - 1]; x2 = xh[t + 1]; xx = x[t]; }
                else if (v == 2) { x0 = x[t]; x1 = x[t + 1]; x2 = x[t - 1]; xx = xh[t]; }
                else { x0 = x[t + 1]; x1 = x[t]; x2 = x[t + 2]; xx = xh[t]; }
                q.xi = (xx - x0) / (x1 - x0);
                q.k = (x2 - x0) / (x1 - x0);
                q.rk = 1.0 / q.k;
                q.r1k = 1.0 / (1.0 - q.k);
                q.rkm1 = 1.0 / (q.k - 1.0);
                return q;
            };
            auto same = [](const QuickCoef& p, const QuickCoef& q) {
                return p.xi == q.xi && p.k == q.k && p.rk == q.rk && p.r1k == q.r1k && p.rkm1 == q.rkm1;
            };
            for (int v = 0; v < 4; v++) {
                const int t0 = v < 2 ? g : g - 1, t1 = v < 2 ? n + g : n + g - 1;
                U->q[a][v] = coef(v, t0);
                for (int t = t0 + 1; t <= t1 && uni; t++) uni = same(coef(v, t), U->q[a][v]);
            }
            U->d[a] = d[g];
            U->dh[a] = dh[g];
            // explicitMomDiff reads the metric one index beyond the interior
            for (int t = g - 1; t <= n + g && uni; t++) uni = d[t] == d[g] && dh[t] == dh[g];
            U->rd[a] = 1. / d[g];
            U->rdh[a] = 1. / dh[g];
        }
        *uniform = uni;
    }
    return PARIS_OK;
}

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
    if (scheme == PARIS_CONV_QUICK) {
        MomTab T;
        QuickUniform U;
        bool exact, uniform;
        PARIS_CHECK(mom_tables(c, &T, &exact, &U, &uniform));
        bool canon = uniform;   // every coefficient set xi = 1/2, k = -1 exactly
        for (int a = 0; a < 3 && canon; a++)
            for (int v = 0; v < 4; v++) canon = canon && U.q[a][v].xi == 0.5 && U.q[a][v].k == -1.0;
        if (canon)
            PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_quick_uniform<true>, cgrid(c->L), cblock(), 0, vel(c),
                           c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, U);
        else if (uniform)
            PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_quick_uniform<false>, cgrid(c->L), cblock(), 0, vel(c),
                           c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, U);
        else if (exact)
            PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_quick<true>, cgrid(c->L), cblock(), 0, vel(c),
                           c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, geo(c),
                           T);
        else
            PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_quick<false>, cgrid(c->L), cblock(), 0, vel(c),
                           c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, geo(c),
                           T);
    } else
        PARIS_LAUNCH_N(c, "mom_convection", c->N, k_conv_onedim, cgrid(c->L), cblock(), 0, vel(c),
                       c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], c->L, c->bnd, geo(c),
                       scheme);
    return PARIS_OK;
}

extern "C" int paris_explicit_mom_diff(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(need(c, {PARIS_FIELD_MU, PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}));
    MomTab T;
    QuickUniform U;
    bool exact, uniform;
    PARIS_CHECK(mom_tables(c, &T, &exact, &U, &uniform));
    if (uniform)
        PARIS_LAUNCH_N(c, "mom_diffusion", c->N, k_mom_diff<true>, cgrid(c->L), cblock(), 0, vel(c),
                       c->fld[PARIS_FIELD_RHO], c->fld[PARIS_FIELD_MU], c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV],
                       c->fld[PARIS_FIELD_DW], c->L, c->bnd, T, U);
    else
        PARIS_LAUNCH_N(c, "mom_diffusion", c->N, k_mom_diff<false>, cgrid(c->L), cblock(), 0, vel(c),
                       c->fld[PARIS_FIELD_RHO], c->fld[PARIS_FIELD_MU], c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV],
                       c->fld[PARIS_FIELD_DW], c->L, c->bnd, T, U);
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
