// plic.cuh -- PLIC geometry in the unit cube and interface normals on the
// device: AL3D, CC3D, FL3D, AREA3D, AREA_CENTROID (vof_functions.f90:43-476)
// and mycs / fd32 / youngs (vofnonmodule.f90:1209-1416).  The operation order
// is the reference's; translation units including this file are compiled
// with -fmad=false so that no FMA changes a rounding.
#pragma once
#include <cuda_runtime.h>

namespace plic {

constexpr double kAthird = 1.0 / 3.0;
constexpr double kEps0 = 1.0e-50;

__device__ inline double dmax1(double a, double b) { return a > b ? a : b; }
__device__ inline double dmin1(double a, double b) { return a < b ? a : b; }

__device__ inline void order3(const double nr[3], double& m1, double& m2, double& m3) {
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double a = dmin1(np1, np2), c = dmax1(np1, np2), b;
    if (np3 < a) { b = a; a = np3; }
    else if (np3 >= c) { b = c; c = np3; }
    else { b = np3; }
    m1 = a; m2 = b; m3 = c;
}

// the trigonometric root of cases (3) and (4b) of AL3D/AREA3D/AREA_CENTROID
__device__ inline double cubic_root(double p, double q, double shift) {
    double pst = sqrt(p);
    double arc = kAthird * acos(q / (p * pst));
    double csarc = cos(arc);
    return pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + shift;
}

// AL3D, vof_functions.f90:43-115
__device__ inline double al3d(const double nr[3], double cc) {
    double m1, m2, m3, r;
    order3(nr, m1, m2, m3);
    double denom = dmax1(6.0 * m1 * m2 * m3, kEps0);
    double cch = dmin1(cc, 1.0 - cc);
    double c01 = m1 * m1 * m1 / denom;
    double c02 = c01 + 0.5 * (m2 - m1) / m3;
    double m12 = m1 + m2, c03;
    if (m12 <= m3) {
        c03 = 0.5 * m12 / m3;
    } else {
        double numer = m3 * m3 * (3.0 * m12 - m3) + m1 * m1 * (m1 - 3.0 * m3) + m2 * m2 * (m2 - 3.0 * m3);
        c03 = numer / denom;
    }
    if (cch <= c01) r = pow(denom * cch, kAthird);
    else if (cch <= c02) r = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
    else if (cch <= c03) r = cubic_root(2.0 * m1 * m2, 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch), m12);
    else if (m12 <= m3) r = m3 * cch + 0.5 * m12;
    else r = cubic_root(m12 * m3 + m1 * m2 - 0.25, 1.5 * m1 * m2 * m3 * (0.5 - cch), 0.5);
    if (cc > 0.5) r = 1.0 - r;
    return r + dmin1(0.0, nr[0]) + dmin1(0.0, nr[1]) + dmin1(0.0, nr[2]);
}

// the five-case polynomial shared by CC3D and FL3D
__device__ inline double cut_fraction(double alh, double m1, double m2, double m3) {
    double m12 = m1 + m2;
    double mm = dmin1(m12, m3);
    double denom = dmax1(6.0 * m1 * m2 * m3, kEps0);
    if (alh <= m1) return alh * alh * alh / denom;
    if (alh <= m2) return 0.5 * alh * (alh - m1) / (m2 * m3) + m1 * m1 * m1 / denom;
    if (alh <= mm) {
        double top = alh * alh * (3.0 * m12 - alh) + m1 * m1 * (m1 - 3.0 * alh);
        return (top + m2 * m2 * (m2 - 3.0 * alh)) / denom;
    }
    if (m12 <= m3) return (alh - 0.5 * m12) / m3;
    double top = alh * alh * (3.0 - 2.0 * alh) + m1 * m1 * (m1 - 3.0 * alh);
    return (top + m2 * m2 * (m2 - 3.0 * alh) + m3 * m3 * (m3 - 3.0 * alh)) / denom;
}

// CC3D, vof_functions.f90:117-173
__device__ inline double cc3d(const double nr[3], double alpha) {
    double m1, m2, m3;
    order3(nr, m1, m2, m3);
    double al = alpha + dmax1(0.0, -nr[0]) + dmax1(0.0, -nr[1]) + dmax1(0.0, -nr[2]);
    al = dmax1(0.0, dmin1(1.0, al));
    double alh = dmin1(al, 1.0 - al);
    double r = cut_fraction(alh, m1, m2, m3);
    if (al > 0.5) r = 1.0 - r;
    return r;
}

// FL3D, vof_functions.f90:175-249
__device__ inline double fl3d(const double nr[3], double alpha, const double x0[3], const double dx[3]) {
    double al = alpha - nr[0] * x0[0] - nr[1] * x0[1] - nr[2] * x0[2];
    al = al + dmax1(0.0, -nr[0] * dx[0]) + dmax1(0.0, -nr[1] * dx[1]) + dmax1(0.0, -nr[2] * dx[2]);
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double almax = np1 * dx[0] + np2 * dx[1] + np3 * dx[2];
    al = dmax1(0.0, dmin1(1.0, al / almax));
    double alh = dmin1(al, 1.0 - al);
    np1 = np1 / almax;
    np2 = np2 / almax;
    np3 = np3 / almax;
    double m1 = dmin1(np1 * dx[0], np2 * dx[1]);
    double m3 = dmax1(np1 * dx[0], np2 * dx[1]);
    double top = np3 * dx[2], m2;
    if (top < m1) { m2 = m1; m1 = top; }
    else if (top >= m3) { m2 = m3; m3 = top; }
    else { m2 = top; }
    double frac = cut_fraction(alh, m1, m2, m3);
    top = dx[0] * dx[1] * dx[2];
    if (al <= 0.5) return frac * top;
    return (1.0 - frac) * top;
}

// AREA3D, vof_functions.f90:251-322
__device__ inline double area3d(const double nr[3], double cc) {
    double m1, m2, m3, al;
    order3(nr, m1, m2, m3);
    double denom = dmax1(2.0 * m1 * m2 * m3, kEps0);
    double cch = dmin1(cc, 1.0 - cc);
    double ccr = dmax1(cch, kEps0);
    double c01 = m1 * m1 * m1 / (3.0 * denom);
    double c02 = c01 + 0.5 * (m2 - m1) / m3;
    double m12 = m1 + m2, c03;
    if (m12 <= m3) {
        c03 = 0.5 * m12 / m3;
    } else {
        double numer = m3 * m3 * (3.0 * m12 - m3) + m1 * m1 * (m1 - 3.0 * m3) + m2 * m2 * (m2 - 3.0 * m3);
        c03 = numer / (3.0 * denom);
    }
    double c00 = sqrt(m1 * m1 + m2 * m2 + m3 * m3);
    if (ccr <= c01) {
        al = pow(3.0 * denom * cch, kAthird);
        return c00 * al * al / denom;
    }
    if (ccr <= c02) {
        al = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
        return c00 * (2.0 * al - m1) / (2.0 * m2 * m3);
    }
    if (ccr <= c03) {
        al = cubic_root(2.0 * m1 * m2, 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch), m12);
        return c00 * (-al * al + m1 * (2.0 * al - m1) + m2 * (2.0 * al - m2)) / denom;
    }
    if (m12 <= m3) return c00 / m3;
    al = cubic_root(m12 * m3 + m1 * m2 - 0.25, 1.5 * m1 * m2 * m3 * (0.5 - cch), 0.5);
    return c00 * (2.0 * al * (1.0 - al) - c00 * c00) / denom;
}

// AREA_CENTROID, vof_functions.f90:344-476
__device__ inline void area_centroid(const double nr[3], double cc, double xc0[3]) {
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double m1, m2, m3, al, ctd0[3], top, bot;
    int ind[3];
    if (np1 <= np2) { m1 = np1; m3 = np2; ind[0] = 0; ind[2] = 1; }
    else { m1 = np2; m3 = np1; ind[0] = 1; ind[2] = 0; }
    if (np3 < m1) { m2 = m1; m1 = np3; ind[1] = ind[0]; ind[0] = 2; }
    else if (np3 >= m3) { m2 = m3; m3 = np3; ind[1] = ind[2]; ind[2] = 2; }
    else { m2 = np3; ind[1] = 2; }
    double denom = dmax1(6.0 * m1 * m2 * m3, kEps0);
    double cch = dmin1(cc, 1.0 - cc);
    double ccr = dmax1(cch, kEps0);
    double c01 = m1 * m1 * m1 / denom;
    double c02 = c01 + 0.5 * (m2 - m1) / m3;
    double m12 = m1 + m2, c03;
    if (m12 <= m3) {
        c03 = 0.5 * m12 / m3;
    } else {
        double numer = m3 * m3 * (3.0 * m12 - m3) + m1 * m1 * (m1 - 3.0 * m3) + m2 * m2 * (m2 - 3.0 * m3);
        c03 = numer / denom;
    }
    if (ccr <= c01) {
        al = pow(denom * cch, kAthird);
        ctd0[0] = kAthird * al / m1;
        ctd0[1] = kAthird * al / m2;
        ctd0[2] = kAthird * al / m3;
    } else if (ccr <= c02) {
        al = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
        top = m1 * m1 + 3. * al * (al - m1);
        bot = dmax1(3. * (2. * al - m1), kEps0);
        ctd0[0] = (3. * al - 2. * m1) / bot;
        ctd0[1] = top / (m2 * bot);
        ctd0[2] = top / (m3 * bot);
    } else if (ccr <= c03) {
        al = cubic_root(2.0 * m1 * m2, 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch), m12);
        bot = 3. * ((al - m2) * (al - m2) + (al - m1) * (al - m1) - al * al);
        top = (al - m2) * (al - m2) * (al - m2) + m1 * m1 * (2. * m1 - 3. * al);
        ctd0[0] = top / (m1 * bot);
        top = (al - m1) * (al - m1) * (al - m1) + m2 * m2 * (2. * m2 - 3. * al);
        ctd0[1] = top / (m2 * bot);
        ctd0[2] = (al - m1 * ctd0[0] - m2 * ctd0[1]) / m3;
    } else if (m12 <= m3) {
        al = m3 * cch + 0.5 * m12;
        ctd0[0] = 0.5;
        ctd0[1] = 0.5;
        ctd0[2] = (al - 0.5 * m12) / m3;
    } else {
        al = cubic_root(m12 * m3 + m1 * m2 - 0.25, 1.5 * m1 * m2 * m3 * (0.5 - cch), 0.5);
        bot = 2.0 * al * (1.0 - al) - (m1 * m1 + m2 * m2 + m3 * m3);
        top = (m1 * m1 * m1 + m2 * m2 * m2 + m3 * m3 * m3) - 3. * al * (m1 * m1 + m2 * m2 + m3 * m3);
        top = kAthird * (top + 3. * al * al - 2. * al * al * al);
        ctd0[0] = (top / m1 - (al - m1) * (al - m1)) / bot;
        ctd0[1] = (top / m2 - (al - m2) * (al - m2)) / bot;
        ctd0[2] = (al - m1 * ctd0[0] - m2 * ctd0[1]) / m3;
    }
    if (cc > 0.5) {
        ctd0[0] = 1.0 - ctd0[0];
        ctd0[1] = 1.0 - ctd0[1];
        ctd0[2] = 1.0 - ctd0[2];
    }
    xc0[ind[0]] = ctd0[0];
    xc0[ind[1]] = ctd0[1];
    xc0[ind[2]] = ctd0[2];
    if (nr[0] < 0.0) xc0[0] = 1.0 - xc0[0];
    if (nr[1] < 0.0) xc0[1] = 1.0 - xc0[1];
    if (nr[2] < 0.0) xc0[2] = 1.0 - xc0[2];
}

// 3x3x3 block c(0:2,0:2,0:2), element (i,j,k) at c[i + 3j + 9k]
#define PC(i, j, k) c[(i) + 3 * (j) + 9 * (k)]

// fd32: mm = -32 grad c, vofnonmodule.f90:1359-1402
__device__ inline void fd32(const double c[27], double mm[3]) {
    double m1, m2;
    m1 = PC(0,0,0) + PC(0,2,0) + PC(0,0,2) + PC(0,2,2) +
         2.0 * (PC(0,0,1) + PC(0,2,1) + PC(0,1,0) + PC(0,1,2)) + 4.0 * PC(0,1,1);
    m2 = PC(2,0,0) + PC(2,2,0) + PC(2,0,2) + PC(2,2,2) +
         2.0 * (PC(2,0,1) + PC(2,2,1) + PC(2,1,0) + PC(2,1,2)) + 4.0 * PC(2,1,1);
    mm[0] = m1 - m2;
    m1 = PC(0,0,0) + PC(0,0,2) + PC(2,0,0) + PC(2,0,2) +
         2.0 * (PC(0,0,1) + PC(2,0,1) + PC(1,0,0) + PC(1,0,2)) + 4.0 * PC(1,0,1);
    m2 = PC(0,2,0) + PC(0,2,2) + PC(2,2,0) + PC(2,2,2) +
         2.0 * (PC(0,2,1) + PC(2,2,1) + PC(1,2,0) + PC(1,2,2)) + 4.0 * PC(1,2,1);
    mm[1] = m1 - m2;
    m1 = PC(0,0,0) + PC(0,2,0) + PC(2,0,0) + PC(2,2,0) +
         2.0 * (PC(0,1,0) + PC(2,1,0) + PC(1,0,0) + PC(1,2,0)) + 4.0 * PC(1,1,0);
    m2 = PC(0,0,2) + PC(0,2,2) + PC(2,0,2) + PC(2,2,2) +
         2.0 * (PC(0,1,2) + PC(2,1,2) + PC(1,0,2) + PC(1,2,2)) + 4.0 * PC(1,1,2);
    mm[2] = m1 - m2;
}

// youngs, vofnonmodule.f90:1404-1416
__device__ inline void youngs(const double c[27], double mm[3]) {
    fd32(c, mm);
    double norm = fabs(mm[0]) + fabs(mm[1]) + fabs(mm[2]);
    mm[0] = mm[0] / norm;
    mm[1] = mm[1] / norm;
    mm[2] = mm[2] / norm;
}

// mycs, vofnonmodule.f90:1209-1357 (NOT_ZERO = single-precision 1.e-30)
__device__ inline void mycs(const double c[27], double mxyz[3]) {
    const double NOT_ZERO = (double)1.e-30f;
    double m1, m2, m[4][3], t0, t1, t2;
    int cn;
    m1 = PC(0,1,0) + PC(0,1,2) + PC(0,0,1) + PC(0,2,1) + PC(0,1,1);
    m2 = PC(2,1,0) + PC(2,1,2) + PC(2,0,1) + PC(2,2,1) + PC(2,1,1);
    m[0][0] = (m1 > m2) ? 1.0 : -1.0;
    m1 = PC(0,0,1) + PC(2,0,1) + PC(1,0,1);
    m2 = PC(0,2,1) + PC(2,2,1) + PC(1,2,1);
    m[0][1] = 0.5 * (m1 - m2);
    m1 = PC(0,1,0) + PC(2,1,0) + PC(1,1,0);
    m2 = PC(0,1,2) + PC(2,1,2) + PC(1,1,2);
    m[0][2] = 0.5 * (m1 - m2);
    m1 = PC(0,0,1) + PC(0,2,1) + PC(0,1,1);
    m2 = PC(2,0,1) + PC(2,2,1) + PC(2,1,1);
    m[1][0] = 0.5 * (m1 - m2);
    m1 = PC(1,0,0) + PC(1,0,2) + PC(2,0,1) + PC(0,0,1) + PC(1,0,1);
    m2 = PC(1,2,0) + PC(1,2,2) + PC(2,2,1) + PC(0,2,1) + PC(1,2,1);
    m[1][1] = (m1 > m2) ? 1.0 : -1.0;
    m1 = PC(1,0,0) + PC(1,1,0) + PC(1,2,0);
    m2 = PC(1,0,2) + PC(1,1,2) + PC(1,2,2);
    m[1][2] = 0.5 * (m1 - m2);
    m1 = PC(0,1,0) + PC(0,1,2) + PC(0,1,1);
    m2 = PC(2,1,0) + PC(2,1,2) + PC(2,1,1);
    m[2][0] = 0.5 * (m1 - m2);
    m1 = PC(1,0,0) + PC(1,0,2) + PC(1,0,1);
    m2 = PC(1,2,0) + PC(1,2,2) + PC(1,2,1);
    m[2][1] = 0.5 * (m1 - m2);
    m1 = PC(0,1,0) + PC(2,1,0) + PC(1,0,0) + PC(1,2,0) + PC(1,1,0);
    m2 = PC(0,1,2) + PC(2,1,2) + PC(1,0,2) + PC(1,2,2) + PC(1,1,2);
    m[2][2] = (m1 > m2) ? 1.0 : -1.0;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        t0 = fabs(m[r][0]) + fabs(m[r][1]) + fabs(m[r][2]);
        m[r][0] = m[r][0] / t0;
        m[r][1] = m[r][1] / t0;
        m[r][2] = m[r][2] / t0;
    }
    t0 = fabs(m[0][0]);
    t1 = fabs(m[1][1]);
    t2 = fabs(m[2][2]);
    cn = 0;
    if (t1 > t0) { t0 = t1; cn = 1; }
    if (t2 > t0) cn = 2;
    fd32(c, m[3]);
    t0 = fabs(m[3][0]) + fabs(m[3][1]) + fabs(m[3][2]) + NOT_ZERO;
    m[3][0] = m[3][0] / t0;
    m[3][1] = m[3][1] / t0;
    m[3][2] = m[3][2] / t0;
    t0 = fabs(m[3][0]);
    t1 = fabs(m[3][1]);
    t2 = fabs(m[3][2]);
    if (t1 > t0) t0 = t1;
    if (t2 > t0) t0 = t2;
    if (fabs(m[cn][cn]) > t0) cn = 3;
    mxyz[0] = m[cn][0];
    mxyz[1] = m[cn][1];
    mxyz[2] = m[cn][2];
}
#undef PC

// FLUX_CENTROID, vof_functions.f90:619-752: the centroid of the part of the
// box [x0, x0 + dx] below the plane nr.x = alpha.  The box goes onto the unit
// cube with positive, sorted coefficients; the centroid below the plane (or
// that of the complement when more than half the box is filled) follows from
// the plane's position in five cases, and is mapped back.
__device__ inline void flux_centroid(const double nr[3], double alpha, const double x0[3], const double dx[3],
                                     double xc0[3]) {
    double al = alpha - nr[0] * x0[0] - nr[1] * x0[1] - nr[2] * x0[2];
    al = al + dmax1(0.0, -nr[0] * dx[0]) + dmax1(0.0, -nr[1] * dx[1]) + dmax1(0.0, -nr[2] * dx[2]);
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    const double almax = np1 * dx[0] + np2 * dx[1] + np3 * dx[2];
    al = dmax1(0.0, dmin1(1.0, al / almax));
    const double alh = dmin1(al, 1.0 - al);
    const double alr = dmax1(alh, kEps0);
    np1 = np1 * dx[0] / almax;
    np2 = np2 * dx[1] / almax;
    np3 = np3 * dx[2] / almax;
    double m1, m2, m3, ctd0[3], frac;
    int ind[3];
    if (np1 <= np2) { m1 = np1; m3 = np2; ind[0] = 0; ind[2] = 1; }
    else { m1 = np2; m3 = np1; ind[0] = 1; ind[2] = 0; }
    if (np3 < m1) { m2 = m1; m1 = np3; ind[1] = ind[0]; ind[0] = 2; }
    else if (np3 >= m3) { m2 = m3; m3 = np3; ind[1] = ind[2]; ind[2] = 2; }
    else { m2 = np3; ind[1] = 2; }
    const double m12 = m1 + m2;
    const double mm = dmin1(m12, m3);
    const double denom = dmax1(6.0 * m1 * m2 * m3, kEps0);
    if (alr <= m1) {
        const double q = 0.25 * alh;
        ctd0[0] = q / m1;
        ctd0[1] = q / m2;
        ctd0[2] = q / m3;
        frac = alh * alh * alh / denom;
    } else if (alr <= m2) {
        const double t1 = (2.0 * alh - m1);
        double t2 = (2.0 * alh * alh - 2.0 * alh * m1 + m1 * m1);
        const double b = 4.0 * (3.0 * alr * alr - 3.0 * alh * m1 + m1 * m1);
        t2 = t1 * t2 / b;
        ctd0[0] = 0.5 - m1 * t1 / b;
        ctd0[1] = t2 / m2;
        ctd0[2] = t2 / m3;
        frac = 0.5 * alh * (alh - m1) / (m2 * m3) + m1 * m1 * m1 / denom;
    } else if (alr <= mm) {
        const double a2 = alh * alh;
        const double t1 = (alh - m1) * (alh - m1) * (alh - m1);
        const double t2 = (alh - m2) * (alh - m2) * (alh - m2);
        const double b = 4.0 * (a2 * alh - t1 - t2);
        ctd0[0] = (a2 * a2 - t1 * (alh + 3.0 * m1) - t2 * (alh - m2)) / (m1 * b);
        ctd0[1] = (a2 * a2 - t1 * (alh - m1) - t2 * (alh + 3.0 * m2)) / (m2 * b);
        ctd0[2] = (a2 * a2 - t1 * (alh - m1) - t2 * (alh - m2)) / (m3 * b);
        const double t3 = alh * alh * (3.0 * m12 - alh) + m1 * m1 * (m1 - 3.0 * alh);
        frac = (t3 + m2 * m2 * (m2 - 3.0 * alh)) / denom;
    } else if (m12 <= m3) {
        const double b = dmax1((2.0 * alh - m12), kEps0);
        ctd0[0] = 0.5 - m1 / (6.0 * b);
        ctd0[1] = 0.5 - m2 / (6.0 * b);
        ctd0[2] = ((3.0 * alh - 2.0 * m12) * b + alh * m12 - m1 * m2) / (6.0 * m3 * b);
        frac = (alh - 0.5 * m12) / m3;
    } else {
        const double s1 = m1 + m2 + m3;
        const double s2 = m1 * m1 + m2 * m2 + m3 * m3;
        const double s3 = m1 * m1 * m1 + m2 * m2 * m2 + m3 * m3 * m3;
        const double s4 = m1 * m1 * m1 * m1 + m2 * m2 * m2 * m2 + m3 * m3 * m3 * m3;
        const double a2 = alh * alh;
        const double b = 4.0 * (2.0 * a2 * alh - 3.0 * a2 * s1 + 3.0 * alh * s2 - s3);
        const double t = 2.0 * a2 * a2 - 4.0 * a2 * alh * s1 + 6.0 * a2 * s2 - 4.0 * alh * s3 + s4;
        ctd0[0] = (t + 4.0 * m1 * (alh - m1) * (alh - m1) * (alh - m1)) / (m1 * b);
        ctd0[1] = (t + 4.0 * m2 * (alh - m2) * (alh - m2) * (alh - m2)) / (m2 * b);
        ctd0[2] = (t + 4.0 * m3 * (alh - m3) * (alh - m3) * (alh - m3)) / (m3 * b);
        const double u1 = alh * alh * (3.0 - 2.0 * alh) + m1 * m1 * (m1 - 3.0 * alh);
        frac = (u1 + m2 * m2 * (m2 - 3.0 * alh) + m3 * m3 * (m3 - 3.0 * alh)) / denom;
    }
    if (al > 0.5) {
        ctd0[0] = (0.5 - frac * (1.0 - ctd0[0])) / (1.0 - frac);
        ctd0[1] = (0.5 - frac * (1.0 - ctd0[1])) / (1.0 - frac);
        ctd0[2] = (0.5 - frac * (1.0 - ctd0[2])) / (1.0 - frac);
    }
    double r[3];
    r[ind[0]] = ctd0[0];
    r[ind[1]] = ctd0[1];
    r[ind[2]] = ctd0[2];
    for (int a = 0; a < 3; a++) {
        if (nr[a] < 0.0) r[a] = 1.0 - r[a];
        xc0[a] = x0[a] + r[a] * dx[a];
    }
}

}  // namespace plic
