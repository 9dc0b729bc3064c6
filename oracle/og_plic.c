/*
 * og_plic.c -- oracle (test infrastructure only): PLIC geometry in the unit
 * cube and interface normals, restated from vof_functions.f90 (Scardovelli)
 * and vofnonmodule.f90 in the same operation order.
 */
#include <math.h>
#include "og.h"

#define ATHIRD (1.0 / 3.0)
#define EPS0 1.0e-50

/* sort |nr| ascending: m1 <= m2 <= m3 (vof_functions.f90:53-65) */
static void og_order3(const double nr[3], double* m1, double* m2, double* m3) {
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double a = og_dmin1(np1, np2), c = og_dmax1(np1, np2), b;
    if (np3 < a) {
        b = a; a = np3;
    } else if (np3 >= c) {
        b = c; c = np3;
    } else {
        b = np3;
    }
    *m1 = a; *m2 = b; *m3 = c;
}

/* AL3D, vof_functions.f90:43-115 */
double og_al3d(const double nr[3], double cc) {
    double m1, m2, m3, r;
    og_order3(nr, &m1, &m2, &m3);
    double denom = og_dmax1(6.0 * m1 * m2 * m3, EPS0);
    double cch = og_dmin1(cc, 1.0 - cc);
    double c01 = m1 * m1 * m1 / denom;
    double c02 = c01 + 0.5 * (m2 - m1) / m3;
    double m12 = m1 + m2, c03;
    if (m12 <= m3) {
        c03 = 0.5 * m12 / m3;
    } else {
        double numer = m3 * m3 * (3.0 * m12 - m3) + m1 * m1 * (m1 - 3.0 * m3) + m2 * m2 * (m2 - 3.0 * m3);
        c03 = numer / denom;
    }
    if (cch <= c01) {
        r = pow(denom * cch, ATHIRD);
    } else if (cch <= c02) {
        r = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
    } else if (cch <= c03) {
        double p = 2.0 * m1 * m2;
        double q = 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        r = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + m12;
    } else if (m12 <= m3) {
        r = m3 * cch + 0.5 * m12;
    } else {
        double p = m12 * m3 + m1 * m2 - 0.25;
        double q = 1.5 * m1 * m2 * m3 * (0.5 - cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        r = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + 0.5;
    }
    if (cc > 0.5) r = 1.0 - r;
    r = r + og_dmin1(0.0, nr[0]) + og_dmin1(0.0, nr[1]) + og_dmin1(0.0, nr[2]);
    return r;
}

/* CC3D, vof_functions.f90:117-173 */
double og_cc3d(const double nr[3], double alpha) {
    double m1, m2, m3, r;
    og_order3(nr, &m1, &m2, &m3);
    double al = alpha + og_dmax1(0.0, -nr[0]) + og_dmax1(0.0, -nr[1]) + og_dmax1(0.0, -nr[2]);
    al = og_dmax1(0.0, og_dmin1(1.0, al));
    double alh = og_dmin1(al, 1.0 - al);
    double m12 = m1 + m2;
    double mm = og_dmin1(m12, m3);
    double denom = og_dmax1(6.0 * m1 * m2 * m3, EPS0);
    if (alh <= m1) {
        r = alh * alh * alh / denom;
    } else if (alh <= m2) {
        r = 0.5 * alh * (alh - m1) / (m2 * m3) + m1 * m1 * m1 / denom;
    } else if (alh <= mm) {
        double top = alh * alh * (3.0 * m12 - alh) + m1 * m1 * (m1 - 3.0 * alh);
        r = (top + m2 * m2 * (m2 - 3.0 * alh)) / denom;
    } else if (m12 <= m3) {
        r = (alh - 0.5 * m12) / m3;
    } else {
        double top = alh * alh * (3.0 - 2.0 * alh) + m1 * m1 * (m1 - 3.0 * alh);
        r = (top + m2 * m2 * (m2 - 3.0 * alh) + m3 * m3 * (m3 - 3.0 * alh)) / denom;
    }
    if (al > 0.5) r = 1.0 - r;
    return r;
}

/* FL3D, vof_functions.f90:175-249 */
double og_fl3d(const double nr[3], double alpha, const double x0[3], const double dx[3]) {
    double al = alpha - nr[0] * x0[0] - nr[1] * x0[1] - nr[2] * x0[2];
    al = al + og_dmax1(0.0, -nr[0] * dx[0]) + og_dmax1(0.0, -nr[1] * dx[1]) + og_dmax1(0.0, -nr[2] * dx[2]);
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double almax = np1 * dx[0] + np2 * dx[1] + np3 * dx[2];
    al = og_dmax1(0.0, og_dmin1(1.0, al / almax));
    double alh = og_dmin1(al, 1.0 - al);
    np1 = np1 / almax;
    np2 = np2 / almax;
    np3 = np3 / almax;
    double m1 = og_dmin1(np1 * dx[0], np2 * dx[1]);
    double m3 = og_dmax1(np1 * dx[0], np2 * dx[1]);
    double top = np3 * dx[2], m2;
    if (top < m1) {
        m2 = m1; m1 = top;
    } else if (top >= m3) {
        m2 = m3; m3 = top;
    } else {
        m2 = top;
    }
    double m12 = m1 + m2;
    double mm = og_dmin1(m12, m3);
    double denom = og_dmax1(6.0 * m1 * m2 * m3, EPS0);
    double frac;
    if (alh <= m1) {
        frac = alh * alh * alh / denom;
    } else if (alh <= m2) {
        frac = 0.5 * alh * (alh - m1) / (m2 * m3) + m1 * m1 * m1 / denom;
    } else if (alh <= mm) {
        top = alh * alh * (3.0 * m12 - alh) + m1 * m1 * (m1 - 3.0 * alh);
        frac = (top + m2 * m2 * (m2 - 3.0 * alh)) / denom;
    } else if (m12 <= m3) {
        frac = (alh - 0.5 * m12) / m3;
    } else {
        top = alh * alh * (3.0 - 2.0 * alh) + m1 * m1 * (m1 - 3.0 * alh);
        frac = (top + m2 * m2 * (m2 - 3.0 * alh) + m3 * m3 * (m3 - 3.0 * alh)) / denom;
    }
    top = dx[0] * dx[1] * dx[2];
    if (al <= 0.5) return frac * top;
    return (1.0 - frac) * top;
}

/* AREA3D, vof_functions.f90:251-322 */
double og_area3d(const double nr[3], double cc) {
    double m1, m2, m3, r, al;
    og_order3(nr, &m1, &m2, &m3);
    double denom = og_dmax1(2.0 * m1 * m2 * m3, EPS0);
    double cch = og_dmin1(cc, 1.0 - cc);
    double ccr = og_dmax1(cch, EPS0);
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
        al = pow(3.0 * denom * cch, ATHIRD);
        r = c00 * al * al / denom;
    } else if (ccr <= c02) {
        al = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
        r = c00 * (2.0 * al - m1) / (2.0 * m2 * m3);
    } else if (ccr <= c03) {
        double p = 2.0 * m1 * m2;
        double q = 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        al = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + m12;
        r = c00 * (-al * al + m1 * (2.0 * al - m1) + m2 * (2.0 * al - m2)) / denom;
    } else if (m12 <= m3) {
        r = c00 / m3;
    } else {
        double p = m12 * m3 + m1 * m2 - 0.25;
        double q = 1.5 * m1 * m2 * m3 * (0.5 - cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        al = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + 0.5;
        r = c00 * (2.0 * al * (1.0 - al) - c00 * c00) / denom;
    }
    return r;
}

/* AREA_CENTROID, vof_functions.f90:344-476 */
void og_area_centroid(const double nr[3], double cc, double xc0[3]) {
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    double m1, m2, m3, al, ctd0[3], top, bot;
    int ind[3];
    if (np1 <= np2) {
        m1 = np1; m3 = np2; ind[0] = 0; ind[2] = 1;
    } else {
        m1 = np2; m3 = np1; ind[0] = 1; ind[2] = 0;
    }
    if (np3 < m1) {
        m2 = m1; m1 = np3; ind[1] = ind[0]; ind[0] = 2;
    } else if (np3 >= m3) {
        m2 = m3; m3 = np3; ind[1] = ind[2]; ind[2] = 2;
    } else {
        m2 = np3; ind[1] = 2;
    }
    double denom = og_dmax1(6.0 * m1 * m2 * m3, EPS0);
    double cch = og_dmin1(cc, 1.0 - cc);
    double ccr = og_dmax1(cch, EPS0);
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
        al = pow(denom * cch, ATHIRD);
        ctd0[0] = ATHIRD * al / m1;
        ctd0[1] = ATHIRD * al / m2;
        ctd0[2] = ATHIRD * al / m3;
    } else if (ccr <= c02) {
        al = 0.5 * (m1 + sqrt(m1 * m1 + 8.0 * m2 * m3 * (cch - c01)));
        top = m1 * m1 + 3. * al * (al - m1);
        bot = og_dmax1(3. * (2. * al - m1), EPS0);
        ctd0[0] = (3. * al - 2. * m1) / bot;
        ctd0[1] = top / (m2 * bot);
        ctd0[2] = top / (m3 * bot);
    } else if (ccr <= c03) {
        double p = 2.0 * m1 * m2;
        double q = 1.5 * m1 * m2 * (m12 - 2.0 * m3 * cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        al = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + m12;
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
        double p = m12 * m3 + m1 * m2 - 0.25;
        double q = 1.5 * m1 * m2 * m3 * (0.5 - cch);
        double pst = sqrt(p);
        double arc = ATHIRD * acos(q / (p * pst));
        double csarc = cos(arc);
        al = pst * (sqrt(3.0 * (1.0 - csarc * csarc)) - csarc) + 0.5;
        bot = 2.0 * al * (1.0 - al) - (m1 * m1 + m2 * m2 + m3 * m3);
        top = (m1 * m1 * m1 + m2 * m2 * m2 + m3 * m3 * m3) - 3. * al * (m1 * m1 + m2 * m2 + m3 * m3);
        top = ATHIRD * (top + 3. * al * al - 2. * al * al * al);
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

/* FLUX_CENTROID, vof_functions.f90:619-752: the centroid of the part of the
 * box [x0, x0+dx] below the plane nr.x = alpha.  The box is mapped onto the
 * unit cube with the coefficients made positive and sorted; the centroid of
 * the region below the plane (or of its complement, when more than half the
 * box is filled) follows from the five cases of the plane's position, and is
 * mapped back. */
void og_flux_centroid(const double nr[3], double alpha, const double x0[3], const double dx[3], double xc0[3]) {
    double al = alpha - nr[0] * x0[0] - nr[1] * x0[1] - nr[2] * x0[2];
    al = al + og_dmax1(0.0, -nr[0] * dx[0]) + og_dmax1(0.0, -nr[1] * dx[1]) + og_dmax1(0.0, -nr[2] * dx[2]);
    double np1 = fabs(nr[0]), np2 = fabs(nr[1]), np3 = fabs(nr[2]);
    const double almax = np1 * dx[0] + np2 * dx[1] + np3 * dx[2];
    al = og_dmax1(0.0, og_dmin1(1.0, al / almax));
    const double alh = og_dmin1(al, 1.0 - al);
    const double alr = og_dmax1(alh, EPS0);
    np1 = np1 * dx[0] / almax;
    np2 = np2 * dx[1] / almax;
    np3 = np3 * dx[2] / almax;
    double m1, m2, m3, ctd0[3], frac;
    int ind[3];
    if (np1 <= np2) {
        m1 = np1; m3 = np2; ind[0] = 0; ind[2] = 1;
    } else {
        m1 = np2; m3 = np1; ind[0] = 1; ind[2] = 0;
    }
    if (np3 < m1) {
        m2 = m1; m1 = np3; ind[1] = ind[0]; ind[0] = 2;
    } else if (np3 >= m3) {
        m2 = m3; m3 = np3; ind[1] = ind[2]; ind[2] = 2;
    } else {
        m2 = np3; ind[1] = 2;
    }
    const double m12 = m1 + m2;
    const double mm = og_dmin1(m12, m3);
    const double denom = og_dmax1(6.0 * m1 * m2 * m3, EPS0);
    if (alr <= m1) {   /* a corner tetrahedron */
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
        const double b = og_dmax1((2.0 * alh - m12), EPS0);
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
    if (al > 0.5) {   /* the filled part is the complement of the computed one */
        ctd0[0] = (0.5 - frac * (1.0 - ctd0[0])) / (1.0 - frac);
        ctd0[1] = (0.5 - frac * (1.0 - ctd0[1])) / (1.0 - frac);
        ctd0[2] = (0.5 - frac * (1.0 - ctd0[2])) / (1.0 - frac);
    }
    xc0[ind[0]] = ctd0[0];
    xc0[ind[1]] = ctd0[1];
    xc0[ind[2]] = ctd0[2];
    if (nr[0] < 0.0) xc0[0] = 1.0 - xc0[0];
    if (nr[1] < 0.0) xc0[1] = 1.0 - xc0[1];
    if (nr[2] < 0.0) xc0[2] = 1.0 - xc0[2];
    xc0[0] = x0[0] + xc0[0] * dx[0];
    xc0[1] = x0[1] + xc0[1] * dx[1];
    xc0[2] = x0[2] + xc0[2] * dx[2];
}

#define C(i, j, k) c[OG_C3(i, j, k)]

/* fd32: mm = -32 grad(c) on the 3x3x3 block, vofnonmodule.f90:1359-1402 */
void og_fd32(const double c[27], double mm[3]) {
    double m1, m2;
    m1 = C(0,0,0) + C(0,2,0) + C(0,0,2) + C(0,2,2) +
         2.0 * (C(0,0,1) + C(0,2,1) + C(0,1,0) + C(0,1,2)) + 4.0 * C(0,1,1);
    m2 = C(2,0,0) + C(2,2,0) + C(2,0,2) + C(2,2,2) +
         2.0 * (C(2,0,1) + C(2,2,1) + C(2,1,0) + C(2,1,2)) + 4.0 * C(2,1,1);
    mm[0] = m1 - m2;
    m1 = C(0,0,0) + C(0,0,2) + C(2,0,0) + C(2,0,2) +
         2.0 * (C(0,0,1) + C(2,0,1) + C(1,0,0) + C(1,0,2)) + 4.0 * C(1,0,1);
    m2 = C(0,2,0) + C(0,2,2) + C(2,2,0) + C(2,2,2) +
         2.0 * (C(0,2,1) + C(2,2,1) + C(1,2,0) + C(1,2,2)) + 4.0 * C(1,2,1);
    mm[1] = m1 - m2;
    m1 = C(0,0,0) + C(0,2,0) + C(2,0,0) + C(2,2,0) +
         2.0 * (C(0,1,0) + C(2,1,0) + C(1,0,0) + C(1,2,0)) + 4.0 * C(1,1,0);
    m2 = C(0,0,2) + C(0,2,2) + C(2,0,2) + C(2,2,2) +
         2.0 * (C(0,1,2) + C(2,1,2) + C(1,0,2) + C(1,2,2)) + 4.0 * C(1,1,2);
    mm[2] = m1 - m2;
}

/* youngs, vofnonmodule.f90:1404-1416 */
void og_youngs(const double c[27], double mm[3]) {
    og_fd32(c, mm);
    double norm = fabs(mm[0]) + fabs(mm[1]) + fabs(mm[2]);
    mm[0] = mm[0] / norm;
    mm[1] = mm[1] / norm;
    mm[2] = mm[2] / norm;
}

/* mycs: Mixed Youngs-Centred normal, vofnonmodule.f90:1209-1357.
 * NOT_ZERO is the single-precision literal 1.e-30 stored in real(8). */
void og_mycs(const double c[27], double mxyz[3]) {
    const double NOT_ZERO = (double)1.e-30f;
    double m1, m2, m[4][3], t0, t1, t2;
    int cn;
    m1 = C(0,1,0) + C(0,1,2) + C(0,0,1) + C(0,2,1) + C(0,1,1);
    m2 = C(2,1,0) + C(2,1,2) + C(2,0,1) + C(2,2,1) + C(2,1,1);
    m[0][0] = (m1 > m2) ? 1.0 : -1.0;
    m1 = C(0,0,1) + C(2,0,1) + C(1,0,1);
    m2 = C(0,2,1) + C(2,2,1) + C(1,2,1);
    m[0][1] = 0.5 * (m1 - m2);
    m1 = C(0,1,0) + C(2,1,0) + C(1,1,0);
    m2 = C(0,1,2) + C(2,1,2) + C(1,1,2);
    m[0][2] = 0.5 * (m1 - m2);

    m1 = C(0,0,1) + C(0,2,1) + C(0,1,1);
    m2 = C(2,0,1) + C(2,2,1) + C(2,1,1);
    m[1][0] = 0.5 * (m1 - m2);
    m1 = C(1,0,0) + C(1,0,2) + C(2,0,1) + C(0,0,1) + C(1,0,1);
    m2 = C(1,2,0) + C(1,2,2) + C(2,2,1) + C(0,2,1) + C(1,2,1);
    m[1][1] = (m1 > m2) ? 1.0 : -1.0;
    m1 = C(1,0,0) + C(1,1,0) + C(1,2,0);
    m2 = C(1,0,2) + C(1,1,2) + C(1,2,2);
    m[1][2] = 0.5 * (m1 - m2);

    m1 = C(0,1,0) + C(0,1,2) + C(0,1,1);
    m2 = C(2,1,0) + C(2,1,2) + C(2,1,1);
    m[2][0] = 0.5 * (m1 - m2);
    m1 = C(1,0,0) + C(1,0,2) + C(1,0,1);
    m2 = C(1,2,0) + C(1,2,2) + C(1,2,1);
    m[2][1] = 0.5 * (m1 - m2);
    m1 = C(0,1,0) + C(2,1,0) + C(1,0,0) + C(1,2,0) + C(1,1,0);
    m2 = C(0,1,2) + C(2,1,2) + C(1,0,2) + C(1,2,2) + C(1,1,2);
    m[2][2] = (m1 > m2) ? 1.0 : -1.0;

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

    og_fd32(c, m[3]);
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
