// limiter.cuh -- minabs / maxabs (paris.f90:3450-3475) and slope_lim
// (modules.f90:177-197): the limited slope of three values for the
// AdvectionScheme ENO, Superbee or WENO, zero for every other scheme.
#pragma once
#include "common.cuh"

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

// interpole3 (modules.f90:199-206): val2 + slope_lim(val1, val2, val3) * delta_x
__device__ inline double interpole3(double v1, double v2, double v3, int scheme, double delta_x) {
    return v2 + slope_lim(v1, v2, v3, scheme) * delta_x;
}
