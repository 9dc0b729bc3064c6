/*
 * og.h -- the CPU oracle: an FP64 C restatement of the PARIS routines on the
 * B200 grid-core path, used ONLY as test infrastructure (the parity checker
 * of tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py).
 * Nothing in the product library links or calls it.
 *
 * Arrays follow the reference layout: real(8) F(imin:imax,jmin:jmax,kmin:kmax)
 * with Ng ghost layers, i fastest.  C index = Fortran index - 1, so the
 * interior is [ng, ng+n) in every direction.  Each routine cites the
 * reference file:line it restates, keeping the Fortran operation order
 * (compiled with -ffp-contract=off so no FMA is introduced).
 *
 * Parity of the oracle is pinned against the reference's own tests:
 *   Tests/PoissonMG (residual < 1e-8, L1 error < 0.1 after 20 V-cycles),
 *   Tests/VOF volumeref.txt / centerofmassref.txt (CIAM, 16^3, tol 1e-4),
 *   Tests/Curvature (sphere curvature, rel. L2 < 4e-2),
 *   Tests/CylinderAdvection reference.txt (DoMOMCONS, staggered Weymouth-Yue,
 *   16 x 16 x 2, 3800 steps: every cell to the five printed digits).
 */
#ifndef PARIS_ORACLE_OG_H
#define PARIS_ORACLE_OG_H

#include <stdint.h>
#include <stdlib.h>
#include "../include/paris_b200.h"

typedef struct og_grid {
    paris_grid_desc d;
    int nx, ny, nz, ng;
    int N[3];               /* interior cells per direction */
    int Nt[3];              /* cells with ghosts per direction */
    long sy, sz;            /* strides of the ghosted layout */
    long ntot;              /* total ghosted cells */
    /* coordinates of the reference (paris.f90:3057-3100), index = Fortran-1 */
    double *x, *xh, *dx, *dxh;
    double *y, *yh, *dy, *dyh;
    double *z, *zh, *dz, *dzh;
} og_grid;

#define OG_IX(g, i, j, k) ((long)(i) + (long)(j) * (g)->sy + (long)(k) * (g)->sz)

static inline double og_dmax1(double a, double b) { return a > b ? a : b; }
static inline double og_dmin1(double a, double b) { return a < b ? a : b; }

og_grid* og_grid_new(const paris_grid_desc* d);
void og_grid_free(og_grid* g);
int og_is_periodic(const og_grid* g, int dir); /* dir 0..2 */

/* ghost_x/y/z with ngh layers (modules.f90:1821-1970) on one rank: periodic
 * wrap, nothing for walls (MPI_PROC_NULL neighbours). */
void og_ghost_dir(const og_grid* g, double* F, int dir, int ngh);
void og_ighost_dir(const og_grid* g, int32_t* F, int dir, int ngh);
void og_do_all_ghost(const og_grid* g, double* F);   /* modules.f90:2062 */
void og_do_all_ighost(const og_grid* g, int32_t* F); /* modules.f90:2076 */

/* geometry (vof_functions.f90) */
double og_al3d(const double nr[3], double cc);
double og_cc3d(const double nr[3], double alpha);
double og_fl3d(const double nr[3], double alpha, const double x0[3], const double dx[3]);
double og_area3d(const double nr[3], double cc);
void og_area_centroid(const double nr[3], double cc, double xc0[3]);
/* normals (vofnonmodule.f90); c is the 3x3x3 block c(0:2,0:2,0:2) in Fortran
 * order: element (i,j,k) at c[i + 3*j + 9*k] */
#define OG_C3(i, j, k) ((i) + 3 * (j) + 9 * (k))
void og_mycs(const double c[27], double m[3]);
void og_fd32(const double c[27], double m[3]);
void og_youngs(const double c[27], double m[3]);
/* FLUX_CENTROID, vof_functions.f90:619-752 */
void og_flux_centroid(const double nr[3], double alpha, const double x0[3], const double dx[3], double xc0[3]);

/* og_vof.c pieces shared with the momentum-conserving sweeps */
void og_setvofbc(const og_grid* g, double* cv, int32_t* fl);          /* SetVOFBC */
void og_flags_and_clip(const og_grid* g, double* c, int32_t* f);      /* get_flags_and_clip */
void og_stencil(const og_grid* g, const double* c, long n, double st[27]);
int og_fit_plane_new(double vof, int d, double a1, double a2, const double st[27], double m[3], double* alpha);
/* swp (vofnonmodule.f90:27-48) along d (0..2) with face velocity us; w2 is
 * the c_mask of the Weymouth-Yue sweep; phase may be NULL */
void og_swp(const og_grid* g, const double* us, double* c, int32_t* f, int d, double dt, double* w1, double* w2,
            double* w3, int32_t* phase);

#endif
