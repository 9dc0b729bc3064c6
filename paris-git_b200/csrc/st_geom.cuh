// st_geom.cuh -- per-cell geometry of the height-function curvature on the
// device: orientation, LineCenter/PlaneAreaCenter, FindCutAreaCentroid,
// NewFindCutAreaCentroid, FindInverseMatrix, parabola_fit(_with_rotation) and
// ind_pos_sorted_add (surface_tension.f90:1056-1702), in the reference's
// operation order (compiled with -fmad=false).
#pragma once
#include "plic.cuh"

namespace stg {

constexpr int kNpos = 28;
constexpr double kEpsGeom = 1e-4;

// orientation: directions sorted by |m|, largest first (0-based)
__device__ inline void orientation(const double m[3], int c[3]) {
    c[0] = 0; c[1] = 1; c[2] = 2;
    for (int i = 1; i <= 2; i++)
        for (int j = 1; j <= 3 - i; j++)
            if (fabs(m[c[j]]) > fabs(m[c[j - 1]])) {
                int t = c[j - 1]; c[j - 1] = c[j]; c[j] = t;
            }
}

__device__ inline double threshold(double z) { return z < 0.0 ? 0.0 : (z > 1.0 ? 1.0 : z); }

__device__ inline void line_center(double dmx, double dmy, double alpha, double& px, double& py) {
    if (dmx < kEpsGeom) { px = 0.5; py = alpha; return; }
    if (dmy < kEpsGeom) { py = 0.5; px = alpha; return; }
    px = 0.; py = 0.0;
    if (alpha >= dmx) { px = px + 1.0; py = py + (alpha - dmx) / dmy; }
    else { px = px + alpha / dmx; }
    if (alpha >= dmy) { py = py + 1.0; px = px + (alpha - dmy) / dmx; }
    else { py = py + alpha / dmy; }
    px = px / 2.0;
    py = py / 2.0;
    px = threshold(px);
    py = threshold(py);
}

__device__ inline void plane_area_center(double dmx, double dmy, double dmz, double alpha, double& px, double& py,
                                         double& pz) {
    double qx, qy, area, b, amax;
    if (dmx < kEpsGeom) { line_center(dmy, dmz, alpha, qx, qy); px = 0.5; py = qx; pz = qy; return; }
    if (dmy < kEpsGeom) { line_center(dmz, dmx, alpha, qx, qy); px = qy; py = 0.5; pz = qx; return; }
    if (dmz < kEpsGeom) { line_center(dmx, dmy, alpha, px, py); pz = 0.5; return; }
    if (alpha < kEpsGeom) { px = 0.0; py = 0.0; pz = 0.0; return; }
    if (alpha > 1.0 - kEpsGeom) { px = 1.0; py = 1.0; pz = 1.0; return; }
    area = alpha * alpha;
    px = area * alpha; py = area * alpha; pz = area * alpha;
    b = alpha - dmx;
    if (b > 0.) { area = area - b * b; px = px - b * b * (2.0 * dmx + alpha); py = py - b * b * b; pz = pz - b * b * b; }
    b = alpha - dmy;
    if (b > 0.0) { area = area - b * b; py = py - b * b * (2.0 * dmy + alpha); px = px - b * b * b; pz = pz - b * b * b; }
    b = alpha - dmz;
    if (b > 0.0) { area = area - b * b; pz = pz - b * b * (2.0 * dmz + alpha); px = px - b * b * b; py = py - b * b * b; }
    amax = alpha - 1.0;
    b = amax + dmx;
    if (b > 0.0) {
        area = area + b * b;
        py = py + b * b * (2.0 * dmy + alpha - dmz);
        pz = pz + b * b * (2.0 * dmz + alpha - dmy);
        px = px + b * b * b;
    }
    b = amax + dmy;
    if (b > 0.0) {
        area = area + b * b;
        px = px + b * b * (2.0 * dmx + alpha - dmz);
        pz = pz + b * b * (2.0 * dmz + alpha - dmx);
        py = py + b * b * b;
    }
    b = amax + dmz;
    if (b > 0.0) {
        area = area + b * b;
        px = px + b * b * (2.0 * dmx + alpha - dmy);
        py = py + b * b * (2.0 * dmy + alpha - dmx);
        pz = pz + b * b * b;
    }
    area = 3.0 * area;
    px = px / (area * dmx);
    py = py / (area * dmy);
    pz = pz / (area * dmz);
    px = threshold(px);
    py = threshold(py);
    pz = threshold(pz);
}

// FindCutAreaCentroid (youngs normal, AL3D, PlaneAreaCenter, cell-centred)
__device__ inline void find_cut_area_centroid(const double st[27], double cc, double cen[3]) {
    double nr[3];
    plic::youngs(st, nr);
    double dmx = nr[0], dmy = nr[1], dmz = nr[2];
    double invx = 1.0, invy = 1.0, invz = 1.0;
    if (dmx < 0.0) { dmx = -dmx; invx = -1.0; }
    if (dmy < 0.0) { dmy = -dmy; invy = -1.0; }
    if (dmz < 0.0) { dmz = -dmz; invz = -1.0; }
    double m[3] = {dmx, dmy, dmz};
    double alpha = plic::al3d(m, cc);
    double px, py, pz;
    plane_area_center(dmx, dmy, dmz, alpha, px, py, pz);
    cen[0] = px * invx; cen[1] = py * invy; cen[2] = pz * invz;
    cen[0] = cen[0] - invx * 0.5;
    cen[1] = cen[1] - invy * 0.5;
    cen[2] = cen[2] - invz * 0.5;
}

// NewFindCutAreaCentroid (youngs normal, AREA_CENTROID, cell-centred)
__device__ inline void new_find_cut_area_centroid(const double st[27], double cc, double cen[3]) {
    double nr[3];
    plic::youngs(st, nr);
    plic::area_centroid(nr, cc, cen);
    cen[0] = cen[0] - 0.5; cen[1] = cen[1] - 0.5; cen[2] = cen[2] - 0.5;
}

// FindInverseMatrix for n = 6 (Gauss-Jordan with the reference's EPSC tests)
__device__ inline bool find_inverse(const double mat[6][6], double inv[6][6], double epsc) {
    const int n = 6;
    double aug[6][12];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 2 * n; j++) aug[i][j] = j < n ? mat[i][j] : (i + n == j ? 1.0 : 0.0);
    for (int k = 0; k < n - 1; k++)
        if (fabs(aug[k][k]) < epsc)
            for (int i = k + 1; i < n; i++)
                if (fabs(aug[i][k]) > epsc)
                    for (int l = 0; l < 2 * n; l++) aug[k][l] = aug[k][l] + aug[i][l];
    for (int k = 0; k < n - 1; k++) {
        if (fabs(aug[k][k]) < epsc) return false;
        for (int j = k + 1; j < n; j++) {
            double m = aug[j][k] / aug[k][k];
            for (int i = k; i < 2 * n; i++) aug[j][i] = aug[j][i] - m * aug[k][i];
        }
    }
    if (fabs(aug[n - 1][n - 1]) < epsc) return false;
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
    return true;
}

__device__ inline bool parabola_fit(const double fit[kNpos][3], const double w[kNpos], int np, double a[6],
                                    double epsc) {
    double m[6][6], inv[6][6], rhs[6];
    for (int i = 0; i < 6; i++) {
        rhs[i] = 0.0;
        a[i] = 0.0;
        for (int j = 0; j < 6; j++) m[i][j] = 0.0;
    }
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
    if (!find_inverse(m, inv, epsc)) return false;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) a[i] = a[i] + inv[i][j] * rhs[j];
    return true;
}

// parabola_fit_with_rotation; bfit rotated in place when do_rotation
__device__ inline bool parabola_fit_rot(double bfit[kNpos][3], const double w[kNpos], const double mv[3], int np,
                                        double a[6], double& ksign, int do_rotation, double epsc) {
    if (do_rotation) {
        double ev[3][3], nrm[3];
        ev[0][2] = mv[0]; ev[1][2] = mv[1]; ev[2][2] = mv[2];
        ksign = 1.0;
        ev[0][0] = mv[2];
        ev[1][0] = 0.0;
        ev[2][0] = -mv[0];
        ev[0][1] = -ev[1][0] * ev[2][2] + ev[2][0] * ev[1][2];
        ev[1][1] = ev[0][0] * ev[2][2] - ev[2][0] * ev[0][2];
        ev[2][1] = -ev[0][0] * ev[1][2] + ev[1][0] * ev[0][2];
        for (int c = 0; c < 3; c++) nrm[c] = sqrt(ev[0][c] * ev[0][c] + ev[1][c] * ev[1][c] + ev[2][c] * ev[2][c]);
        for (int i = 0; i < 3; i++)
            for (int c = 0; c < 3; c++) ev[i][c] = ev[i][c] / nrm[c];
        for (int q = 0; q < np; q++) {
            double f0 = bfit[q][0], f1 = bfit[q][1], f2 = bfit[q][2];
            for (int i = 0; i < 3; i++) bfit[q][i] = ev[0][i] * f0 + ev[1][i] * f1 + ev[2][i] * f2;
        }
    } else {
        ksign = copysign(1.0, mv[2]);
    }
    return parabola_fit(bfit, w, np, a, epsc);
}

// ind_pos_sorted_add: origin first, then the points farther than 1/2 from
// every earlier point of the input list
__device__ inline int ind_pos_sorted_add(const double cen[3], const double pts[kNpos][3], double bp[kNpos][3], int n) {
    bp[0][0] = cen[0]; bp[0][1] = cen[1]; bp[0][2] = cen[2];
    if (n < 2) return n;
    int ni = 2;
    bp[1][0] = pts[0][0]; bp[1][1] = pts[0][1]; bp[1][2] = pts[0][2];
    for (int j = 1; j < n; j++) {
        bool reject = false;
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

}  // namespace stg
