/*
 * og_debris.c -- oracle of clean_debris (vofmodules.f90:2087-2234), test
 * infrastructure only.  Arrays are ghosted, C index = Fortran index - 1
 * (interior [ng, ng+n)), and the loops keep the reference's order: method 3
 * updates cvof and vof_flag in place in the k, j, i order of the reference,
 * so a cell sees the cells cleaned before it in the same sweep.
 *
 *   method 1: phase_id = +1 where cvof > 0.5 (all cells, ghosts included),
 *             -1 elsewhere; an interior cell whose (2n+1)^3 neighbourhood
 *             holds only its own phase is set to that pure phase;
 *   method 2: a cell below 0.1 whose neighbourhood sum is below 0.3 is set
 *             to 0, one above 0.9 whose sum is within 0.3 of the box size to 1;
 *   method 3: a mixed cell with fewer than 6 mixed cells among its 27 is set
 *             to its phase (vof_phase: cvof >= 0.5 - EPSC); sweeps repeat,
 *             with do_all_ghost, get_flags_and_clip and get_vof_phase between
 *             them, until a sweep cleans nothing (the count of cleaned cells
 *             accumulates over the sweeps, as in the reference) or 11 sweeps.
 * The neighbourhood extends nb cells in each direction, none in z when
 * Nz == 2 (the reference's 2-D case).
 */
#include <string.h>

#include "og.h"

#define IX(i, j, k) OG_IX(g, i, j, k)

/* get_flags_and_clip on the whole array (vofmodules.f90:549-571) */
static void flags_clip_all(const og_grid* g, double* c, int32_t* f, double epsc) {
    for (long n = 0; n < g->ntot; n++) {
        if (c[n] <= epsc) { f[n] = 0; c[n] = 0.0; }
        else if (c[n] >= 1.0 - epsc) { f[n] = 1; c[n] = 1.0; }
        else f[n] = 2;
    }
}

int og_clean_debris(const paris_grid_desc* desc, double* cvof, int32_t* flag, int method, int nb, int* sweeps_out) {
    og_grid* g = og_grid_new(desc);
    if (!g) return PARIS_BAD_ARGS;
    const int is = g->ng, ie = g->ng + g->nx - 1, js = g->ng, je = g->ng + g->ny - 1, ks = g->ng,
              ke = g->ng + g->nz - 1;
    const int ni = nb, nj = nb, nk = g->nz == 2 ? 0 : nb;
    int sweeps = 0;
    if (method == 1 || method == 2) {
        int8_t* cf = calloc(g->ntot, 1);
        int8_t* ph = malloc(g->ntot);
        for (long n = 0; n < g->ntot; n++) ph[n] = cvof[n] > 0.5 ? 1 : -1;
        if (method == 1) {
            for (int i = is; i <= ie; i++)
                for (int j = js; j <= je; j++)
                    for (int k = ks; k <= ke; k++) {
                        long n = IX(i, j, k);
                        cf[n] = ph[n];
                        int stop = 0;
                        for (int i0 = -ni; i0 <= ni && !stop; i0++)
                            for (int j0 = -nj; j0 <= nj && !stop; j0++)
                                for (int k0 = -nk; k0 <= nk && !stop; k0++)
                                    if (ph[n] * ph[IX(i + i0, j + j0, k + k0)] == -1) { cf[n] = 0; stop = 1; }
                    }
        } else {
            const double cvof_min = 0.1, sum_cvof_min = 0.3;
            const double sum1 = (double)((1 + ni * 2) * (1 + nj * 2) * (1 + nk * 2));
            for (int i = is; i <= ie; i++)
                for (int j = js; j <= je; j++)
                    for (int k = ks; k <= ke; k++) {
                        double sum_cvof = 0.0;
                        for (int i0 = -ni; i0 <= ni; i0++)
                            for (int j0 = -nj; j0 <= nj; j0++)
                                for (int k0 = -nk; k0 <= nk; k0++) sum_cvof = sum_cvof + cvof[IX(i + i0, j + j0, k + k0)];
                        long n = IX(i, j, k);
                        if (cvof[n] < cvof_min && sum_cvof < sum_cvof_min) cf[n] = -1;
                        if (cvof[n] > 1.0 - cvof_min && sum_cvof > sum1 - sum_cvof_min) cf[n] = 1;
                    }
        }
        for (int i = is; i <= ie; i++)
            for (int j = js; j <= je; j++)
                for (int k = ks; k <= ke; k++) {
                    long n = IX(i, j, k);
                    if (cf[n] == -1 && cvof[n] > 0.0) cvof[n] = 0.0;
                    else if (cf[n] == 1 && cvof[n] < 1.0) cvof[n] = 1.0;
                }
        free(cf);
        free(ph);
        sweeps = 1;
    } else if (method == 3) {
        const double epsc = desc->epsc;
        int all_clean = 0, itr = 0, cleaned_mix = 0;
        while (!all_clean && itr <= 10) {
            itr++;
            for (int k = ks; k <= ke; k++)
                for (int j = js; j <= je; j++)
                    for (int i = is; i <= ie; i++) {
                        long n = IX(i, j, k);
                        if (flag[n] != 2) continue;
                        int nposit = 0;
                        for (int m = -1; m <= 1; m++)
                            for (int q = -1; q <= 1; q++)
                                for (int l = -1; l <= 1; l++)
                                    if (flag[IX(i + m, j + q, k + l)] == 2) nposit++;
                        if (nposit < 6) {
                            if (!(cvof[n] < 0.5 - epsc)) { cvof[n] = 1.0; flag[n] = 1; }
                            else { cvof[n] = 0.0; flag[n] = 0; }
                            cleaned_mix++;
                        }
                    }
            if (cleaned_mix == 0) all_clean = 1;
            if (!all_clean) {
                og_do_all_ghost(g, cvof);
                flags_clip_all(g, cvof, flag, epsc);
            }
        }
        sweeps = itr;
    } else {
        og_grid_free(g);
        return PARIS_BAD_ARGS;
    }
    if (sweeps_out) *sweeps_out = sweeps;
    og_grid_free(g);
    return PARIS_OK;
}
