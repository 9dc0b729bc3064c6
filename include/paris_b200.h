/*
 * paris_b200.h -- C-ABI of the B200 (sm_100a) grid core of the PARIS two-phase
 * flow solver: split PLIC VOF advection, height-function curvature with the CSF
 * surface-tension force, and the variable-density multigrid pressure projection.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (PARIS_OK on success).  Host arrays use the reference's Fortran layout:
 * real(8) arrays dimensioned (imin:imax, jmin:jmax, kmin:kmax) with Ng ghost
 * layers, i fastest, exactly as the module globals of PARIS are allocated
 * (paris.f90:3016-3031, vofmodules.f90:430).  The matrix A has the layout
 * A(is:ie, js:je, ks:ke, 8) (modules.f90:2729).  Fields live on the device
 * between calls; upload/download move them to and from the Fortran arrays.
 *
 * A Fortran driver binds these with ISO_C_BINDING, through an interface
 * module that keeps the original subroutine names and signatures.
 */
#ifndef PARIS_B200_H
#define PARIS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PARIS_OK             0
#define PARIS_NOT_CONVERGED  1  /* solver hit maxit: the reference sets it=maxit+1 and warns (MGsolver.f90:402) */
#define PARIS_NAN_DETECTED   2  /* NaN in A or p (newsolver.f90:138-173 catch_divergence) */
#define PARIS_BAD_ARGS       3  /* invalid sizes, options or pointers */
#define PARIS_CUDA_ERROR     4  /* a CUDA runtime call failed */
#define PARIS_SETUP_ERROR    5  /* check_poisson_setup failed (newsolver.f90:275-344) */
#define PARIS_NO_DEVICE      6  /* no usable CUDA device */
#define PARIS_CFL_TOO_LARGE  7  /* get_cfl_and_check: CFL above cflmax_allowed (paris.f90:1072) */

/* ---- boundary conditions ----------------------------------------------- */
/* BDRY_COND of the &PARAMETERS namelist (order x- y- z- x+ y+ z+).          */
#define PARIS_BC_WALL      0
#define PARIS_BC_PERIODIC  1
#define PARIS_BC_SHEAR     2   /* a wall for the pressure equation (modules.f90:925) */
/* vofbdry_cond of &VOFPARAMETERS (SetVOFBC, vofmodules.f90:1694-1825).      */
#define PARIS_VOFBC_DRY       0
#define PARIS_VOFBC_WET       1
#define PARIS_VOFBC_JET       2   /* 'jet': x- only; the first ghost layer is inject(j,k) of the
                                     inject_type below, the second keeps its value (vofmodules.f90:1716-1718,1758-1760,1797-1811) */
#define PARIS_VOFBC_PERIODIC  3
#define PARIS_VOFBC_OUTFLOW   4
#define PARIS_VOFBC_90DEG     5   /* '90deg': the first ghost layer copies the adjacent cell, the
                                     second keeps its value (vofmodules.f90:1719-1720,1771-1790) */

/* VOF_advect of &VOFPARAMETERS */
#define PARIS_ADVECT_CIAM  0   /* 'CIAM'      -> swpz (vofnonmodule.f90:126)  */
#define PARIS_ADVECT_WY    1   /* 'Dick_Yue'  -> swpr (vofnonmodule.f90:664)  */

/* DensMean / ViscMean flags of linfunc (vofmodules.f90:171) */
#define PARIS_MEAN_ARITH  101  /* ArithMean, vofmodules.f90:109 */
#define PARIS_MEAN_HARM   102  /* HarmMean,  vofmodules.f90:110 */

/* ---- grid and physical parameters -------------------------------------- */
typedef struct paris_grid_desc {
    int32_t nx, ny, nz;          /* Nx, Ny, Nz: interior cells (one rank, no MPI split); at
                                    least 4 each, or Nz = 2 for a two-dimensional run    */
    int32_t ng;                  /* Ng of the host arrays; must be 2 (modules.f90 Ng) */
    int32_t bdry_cond[6];        /* PARIS_BC_*, order x- y- z- x+ y+ z+ */
    int32_t vofbdry_cond[6];     /* PARIS_VOFBC_* */
    double  xlength, ylength, zlength;  /* XLENGTH/YLENGTH/ZLENGTH; uniform grid (xform=0) */
    int32_t vof_advect;          /* PARIS_ADVECT_* */
    int32_t dens_mean;           /* PARIS_MEAN_* used by paris_linfunc for rho */
    int32_t visc_mean;           /* PARIS_MEAN_* used by paris_linfunc for mu */
    int32_t nfilter;             /* 0 or 1 (27-point filter in linfunc) */
    double  rho1, rho2;          /* RHO1 (cvof=0), RHO2 (cvof=1) */
    double  mu1, mu2;            /* MU1, MU2 */
    double  sigma;               /* SIGMA */
    double  epsc;                /* EPSC, default 1e-12 */
    int32_t nrelax;              /* smoothing sweeps per level of the reference MG (default 3) */
    int32_t sym_mg;              /* sym_MG flag of the reference MG */
    int32_t device;              /* CUDA device ordinal */
    int32_t mixed_heights;       /* mixed_heights flag of the curvature (default 1) */
    int32_t use_full_heights;    /* use_full_heights flag (default 1) */
    int32_t do_rotation;         /* do_rotation flag of the paraboloid fit (default 0) */
    int32_t inject_type;         /* inject_type of &PARAMETERS (modules.f90:872); with a 'jet' VOF
                                    condition the first ghost layer at x- is liquid where
                                    2 or 4: (y-jetcenter_yc)^2 + (z-jetcenter_zc)^2 < radius_liq_inject^2,
                                    3: y-jetcenter_yc <= radius_liq_inject,
                                    5: radius_gas_inject < y-jetcenter_yc < radius_liq_inject,
                                    and gas otherwise (vofmodules.f90:1797-1811)                  */
    int32_t reserved[3];
    double  jetcenter_yc, jetcenter_zc;           /* modules.f90:397 */
    double  radius_liq_inject, radius_gas_inject; /* modules.f90:395 */
} paris_grid_desc;

typedef struct paris_ctx* paris_handle_t;

/* ---- fields ------------------------------------------------------------ */
#define PARIS_FIELD_CVOF      0   /* cvof, cell centres */
#define PARIS_FIELD_U         1   /* u at faces i+1/2 */
#define PARIS_FIELD_V         2
#define PARIS_FIELD_W         3
#define PARIS_FIELD_RHO       4
#define PARIS_FIELD_P         5
#define PARIS_FIELD_DU        6   /* momentum source du,dv,dw (surfaceForce output) */
#define PARIS_FIELD_DV        7
#define PARIS_FIELD_DW        8
#define PARIS_FIELD_KAPPA     9   /* curvature (cell units, 2e6 = uncomputed) */
#define PARIS_FIELD_MU       10
#define PARIS_FIELD_VOF_FLAG 11   /* integer vof_flag (host int32) */
#define PARIS_FIELD_A        12   /* A(is:ie,js:je,ks:ke,8), no ghosts */
#define PARIS_FIELD_HEIGHT   13   /* height(imin:imax,...,6) */
#define PARIS_FIELD_VOF_PHASE 14  /* integer vof_phase (host int32) */
#define PARIS_FIELD_USTAR    15   /* caller scratch face fields, e.g. the predicted  */
#define PARIS_FIELD_VSTAR    16   /* velocity u* kept on the device between steps    */
#define PARIS_FIELD_WSTAR    17
#define PARIS_FIELD_MOMENTUM 18   /* momentum of the momentum-conserving sweeps (DoMOMCONS), */
                                  /* zero when first used, kept between calls               */
#define PARIS_NFIELDS        19

/* ---- life cycle (replaces the allocations of initialize/initialize_VOF,
 *      paris.f90:3016-3031 and init_MG, MGsolver.f90:34-65) --------------- */
int paris_gpu_init(const paris_grid_desc* desc, paris_handle_t* out);
int paris_gpu_finalize(paris_handle_t h);
/* Copy one field between the device mirror and a host array in the reference
 * layout, ghost layers included, as they stand.  VOF_FLAG/VOF_PHASE take
 * int32 arrays, every other field real(8).                                 */
int paris_gpu_upload(paris_handle_t h, int32_t field, const void* host);
int paris_gpu_download(paris_handle_t h, int32_t field, void* host);
/* Device-to-device copy of one real(8) field into another (ghosts included). */
int paris_gpu_copy_field(paris_handle_t h, int32_t dst_field, int32_t src_field);
/* Set every element of a real(8) field (ghosts included) to value. */
int paris_gpu_fill_field(paris_handle_t h, int32_t field, double value);
/* Block until all work queued on the handle's stream has finished. */
int paris_gpu_sync(paris_handle_t h);
/* Asynchronous transfers of real(8) fields, for drivers that overlap their
 * host I/O with the steps.  paris_gpu_upload_async starts copying the host
 * array (pin it for the copy to run concurrently) into a device staging copy
 * of the field on a transfer stream and returns; paris_gpu_upload_commit is
 * the point in the handle's work from which the field holds those values
 * (the handle's stream waits there for the copy).  Issue the upload early
 * and the commit late to overlap the copy with the work in between.
 * paris_gpu_download_async snapshots the field as the handle's work issued
 * before the call left it and copies it to the host on a second transfer
 * stream.  Host arrays must stay valid, and a download's must not be read,
 * until paris_gpu_sync_transfers returns.  No counterpart in the reference
 * (its arrays live on the host).  Flags, A and heights are transferred with
 * the synchronous calls only (PARIS_BAD_ARGS here).                        */
int paris_gpu_upload_async(paris_handle_t h, int32_t field, const void* host);
int paris_gpu_upload_commit(paris_handle_t h, int32_t field);
int paris_gpu_download_async(paris_handle_t h, int32_t field, void* host);
int paris_gpu_sync_transfers(paris_handle_t h);
/* The cudaStream_t the handle issues all work on (as void*). */
void* paris_gpu_stream(paris_handle_t h);
/* Device pointer of a field (interior-only, i fastest; A: 8 components). */
void* paris_gpu_field_ptr(paris_handle_t h, int32_t field);
/* Text of the last error recorded on the handle (never NULL). */
const char* paris_gpu_last_error(paris_handle_t h);
/* Number of kernels this handle launched since creation (launch counter). */
int64_t paris_gpu_launch_count(paris_handle_t h);
/* Per-kernel timing with CUDA events on the handle's stream: enable = 1
 * clears the table and brackets every following launch with two events,
 * enable = 0 stops.  The report is one line per kernel,
 * "name<TAB>launches<TAB>total_ms<TAB>cells", cells being the sum over the
 * launches of the grid cells each launch processed.  Returns the bytes
 * needed (including the terminating 0); writes at most len bytes.          */
int paris_gpu_profile(paris_handle_t h, int32_t enable);
int64_t paris_gpu_profile_report(paris_handle_t h, char* buf, int64_t len);

/* ---- VOF (replaces vofsweeps, vofmodules.f90:1340-1361, with
 *      swp/swpz/swpr, vofnonmodule.f90:27-48,126-237,664-754) ------------ */
int paris_vof_sweeps(paris_handle_t h, int32_t tswap, double dt);
/* linfunc(field,a1,a2,MeanFlag), vofmodules.f90:171-218; which = RHO or MU */
int paris_linfunc(paris_handle_t h, int32_t which);
/* Initial condition: union of spheres by ls2vof_refined
 * (vofmodules.f90:1195-1293 with shapes2ls :973-993).                      */
int paris_init_spheres(paris_handle_t h, int32_t nb, const double* xc, const double* yc,
                       const double* zc, const double* rad, int32_t refinement);

/* ---- heights, curvature, CSF ------------------------------------------- */
/* get_all_heights, surface_tension.f90:185-260 */
int paris_get_all_heights(paris_handle_t h);
/* get_all_curvatures, surface_tension.f90:620-755; kappa_host may be NULL  */
int paris_get_all_curvatures(paris_handle_t h, double* kappa_host);
/* surfaceForce(du,dv,dw,rho), paris.f90:2862-2957 (adds to du,dv,dw) */
int paris_surface_force(paris_handle_t h);

/* ---- momentum predictor ---------------------------------------------- */
#define PARIS_CONV_QUICK     0   /* AdvectionScheme = 'QUICK'    */
#define PARIS_CONV_ENO       1   /* AdvectionScheme = 'ENO'      */
#define PARIS_CONV_SUPERBEE  2   /* AdvectionScheme = 'Superbee' */
#define PARIS_CONV_WENO      3   /* AdvectionScheme = 'WENO'     */
/* momentumConvection, paris.f90:1957-1984 (QUICK :2288-2414; ENO, Superbee,
 * WENO: momentumConvection_onedim :1991-2071): DU, DV, DW are assigned on
 * the updated faces from U, V, W (ghosts filled)                          */
int paris_momentum_convection(paris_handle_t h, int32_t scheme);
/* explicitMomDiff(u,v,w,rho,mu,du,dv,dw), paris.f90:2757-2808 (adds)      */
int paris_explicit_mom_diff(paris_handle_t h);
/* volumeForce(rho,rho1,rho2,dpdx,dpdy,dpdz,BuoyancyCase,fx,fy,fz,gx,gy,gz,
 * du,dv,dw,rho_ave), paris.f90:2813-2860 with fx = fy = fz = 0 (adds)     */
int paris_volume_force(paris_handle_t h, double dpdx, double dpdy, double dpdz, int32_t buoyancy_case,
                       double gx, double gy, double gz, double rho_ave);
/* u = u + dt*du (whole arrays), paris.f90:442-444                         */
int paris_advance_velocity(paris_handle_t h, double dt);
/* SetVelocityBC(u,v,w,...) for walls (bdry_cond 0) and periodic (1)
 * boundaries, modules.f90:951-973,1061-1105, then do_ghost_vector
 * (modules.f90:1628).  wall_vel: WallVel(6,3) in Fortran order, face f
 * (1 x-, 2 x+, 3 y-, 4 y+, 5 z-, 6 z+) component c at (f-1)+6*(c-1);
 * NULL for resting walls.  Other boundary types return PARIS_BAD_ARGS.    */
int paris_set_velocity_bc(paris_handle_t h, const double* wall_vel);
/* vofandmomsweepsstaggered(tswap, t), vofmodules.f90:1536-1692 (DoMOMCONS,
 * called before vofsweeps, paris.f90:303-305): for each velocity component,
 * the momentum is formed on a staggered (staggered = 1: get_momentum_staggered,
 * :1396-1449) or centred (0: get_momentum_centered, :1363-1394) control
 * volume, advected with a copy of the volume fraction by the three split
 * CIAM or Weymouth-Yue sweeps in the order of MOD(tswap,3) (swpmom_stg/swp_stg,
 * vofnonmodule.f90:50-116,239-631,757-1139, or swpmom/swp), and DU/DV/DW are
 * replaced by (mom/rho - u)/dt where the advected fraction is mixed
 * (get_velocity_from_momentum_*, vofmodules.f90:1451-1534).  lin_interp:
 * LinInterp (linear momentum profile across the flux volumes, staggered
 * only); scheme: PARIS_CONV_* of AdvectionScheme for interpole3.  CVOF and
 * VOF_FLAG are read, MOMENTUM is kept.  Boundaries: periodic and walls
 * (SetMomentumBC, modules.f90:1329-1625; wall_vel as for
 * paris_set_velocity_bc); others return PARIS_BAD_ARGS.                  */
int paris_vof_mom_sweeps(paris_handle_t h, int32_t tswap, double dt, int32_t staggered, int32_t lin_interp,
                         int32_t scheme, const double* wall_vel);

/* ---- time-step control and flow statistics ---------------------------- */
/* TimeStepSize(dt, vof_phase), paris.f90:968-1041, for a run without a free
 * surface: vmax = max over the interior of sqrt(u^2+v^2+w^2) taken at the
 * same (i,j,k) of the three face fields, vmax_phys = max(1e-3, u_inject)
 * (u_inject = max(ugas_inject, uliq_inject), 0 without injection),
 * dt = min(cfl * h / max(vmax_phys, vmax), max_dt) with h = minval(dx).
 * vmax_out may be NULL.                                                      */
int paris_time_step_size(paris_handle_t h, double cfl, double max_dt, double u_inject, double* dt,
                         double* vmax_out);
/* get_cfl_and_check(dt), paris.f90:1045-1074: cfl = vmax*dt/h; returns
 * PARIS_CFL_TOO_LARGE (with *cfl written) when cfl > cflmax_allowed (the
 * reference stops with "CFL too large"; cflmax_allowed defaults to 0.5).    */
int paris_get_cfl_and_check(paris_handle_t h, double dt, double cflmax_allowed, double* cfl);

#define PARIS_NSTATS 25
#define PARIS_STATS_RISING_BUBBLE   1   /* test_risingbubble  */
#define PARIS_STATS_PHASE_INVERSION 2   /* test_PhaseInversion */
#define PARIS_STATS_TURB            4   /* test_turb           */
typedef struct paris_stats_opts {
    /* volumeForce arguments of the step the statistics follow: calcStats
     * sums fx, fy, fz = -dpdx + (rho_face - rro)*g as volumeForce left them */
    double  dpdx, dpdy, dpdz;
    double  gx, gy, gz;
    double  rho_ave;             /* rro of BuoyancyCase 3 */
    int32_t buoyancy_case;       /* BuoyancyCase 0..3 */
    int32_t force_valid;         /* 0: fx = fy = fz = 0 (before the first step) */
    int32_t test_flags;          /* PARIS_STATS_* */
    int32_t reserved[3];
} paris_stats_opts;
/* calcStats, paris.f90:1116-1267: stats[0..24] = stats(1:25) (1 wall shear
 * on y, 2 <u>, 3-5 <f>, 6 <rho>, 7 <p>, 8-9 momentum, 10 liquid volume
 * fraction, 11 x centre of mass, 12-13 kinetic energy per phase, 14-15
 * y-momentum per phase, 17-18 inflow/outflow pressure, 19 PLIC interface
 * area, 20-21 potential energy, 22-23 enstrophy per phase, 24 rise velocity
 * or top-layer fraction, 25 mixed-cell count) from the device fields, after
 * the velocity BCs of the step.  Column 9 uses uold, which the reference
 * keeps only for itime_scheme 2; with the explicit scheme it is zero, and it
 * is zero here.  Sums are block partials added in a fixed order, so they are
 * reproducible but not in the reference's loop order.  opts NULL: no force,
 * no test flags.                                                             */
int paris_calc_stats(paris_handle_t h, const paris_stats_opts* opts, double* stats);

/* ---- pressure projection ---------------------------------------------- */
/* SetPressureBC + SetupPoisson + Poisson_BCs + check_poisson_setup,
 * modules.f90:916-949,2722-2892; newsolver.f90:275-344                     */
int paris_setup_poisson(paris_handle_t h, double dt, double volume_source);
/* Setup_testMG, modules.f90:3160-3192 (known-answer RHS)                   */
int paris_setup_test_mg(paris_handle_t h);

#define PARIS_MG_REFERENCE  0  /* FP64, the reference V-cycle step for step (MGsolver.f90:253-405) */
#define PARIS_MG_FP64       1  /* FP64 V(nu1,nu2) cycles in an FP64 defect-correction loop     */
#define PARIS_MG_MIXED      2  /* FP32 V(nu1,nu2) cycles in an FP64 defect-correction loop     */

typedef struct paris_solve_opts {
    double  max_error;   /* stop when the residual norm (order `norm`, RMS) < max_error:
                            the reference's maxError/MaxDt (paris.f90:499)              */
    double  rel_tol;     /* if > 0, stop instead when ||r||_2 / ||b||_2 < rel_tol        */
    double  beta;        /* BETA, relaxation factor of RedBlackRelax (newsolver.f90:229); the
                            FP64/MIXED modes over-relax their red-black smoother by it too:
                            x + beta (x_GS - x); 1 = Gauss-Seidel, <= 0 taken as 1        */
    int32_t maxit;       /* MAXIT                                                         */
    int32_t norm;        /* ResNormOrderPressure: 1 or 2                                  */
    int32_t mode;        /* PARIS_MG_*                                                    */
    int32_t nu1, nu2;    /* pre/post smoothing sweeps of the FP64/MIXED cycles (2,2)      */
    int32_t pcg;         /* FP64/MIXED: 1 = use the V-cycle as a CG preconditioner        */
    int32_t nu_coarse;   /* FP64/MIXED: if > 0, the pre- and post-smoothing sweeps on the
                            levels from coarse_from down (nu1/nu2 above them)              */
    int32_t coarse_from; /* the first level (0 = finest) that takes nu_coarse; 0 taken as 1 */
    int32_t coarse_to;   /* the last level that takes nu_coarse (0: every level below coarse_from) */
    int32_t reserved;    /* 0                                                              */
    double  beta_coarse; /* FP64/MIXED: if > 0, the smoother's relaxation factor on every level
                            below the finest (beta on the finest); <= 0: beta everywhere   */
} paris_solve_opts;

typedef struct paris_solve_result {
    int32_t it;          /* cycles run; maxit+1 when not converged (reference convention) */
    int32_t reserved;
    double  res;         /* tres2: residual in the reference norm at exit                 */
    double  rel_res;     /* ||r||_2 / ||b||_2 at exit                                     */
    double  res0;        /* residual norm before the first cycle                          */
} paris_solve_result;

/* NewSolver(A,p,maxError,beta,maxit,it,ierr,norm), newsolver.f90:34-57 ->
 * NewSolverMG, MGsolver.f90:346-405.  Solves for p (device field P) with the
 * matrix built by paris_setup_poisson (or uploaded as PARIS_FIELD_A).       */
int paris_new_solver(paris_handle_t h, const paris_solve_opts* opts, paris_solve_result* res);
/* calcResiduals, modules.f90:3313-3387: out[0..2] = L1, L2, Linf */
int paris_calc_residuals(paris_handle_t h, double* out3);
/* get_MGtest_err, MGsolver.f90:407-426 (L1 error vs sin*sin*sin / L1 ref) */
int paris_mg_test_err(paris_handle_t h, double* err);
/* project_velocity, paris.f90:882-909 */
int paris_project_velocity(paris_handle_t h, double dt);

/* calcResiduals without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory, e.g. a
 * driver whose device memory is all owned by its own pool or by another
 * runtime, or one held to a fixed memory budget.  A_dev: A(is:ie,js:je,ks:ke,8)
 * and p_dev: p(imin:imax,jmin:jmax,kmin:kmax) (ng ghost layers), both already
 * on the current device in the reference layout; out3 (host) receives L1, L2,
 * Linf as calcResiduals.  stream: a cudaStream_t or NULL.  Scratch is a fixed
 * 1.5 MiB device array held by every GPU that loads the library: grids above
 * 16,777,216 interior cells are rejected (PARIS_BAD_ARGS).  All calls share
 * that array, so calls that overlap on the GPU race.  Every call looks up the
 * array's device address in the current context (no allocation); with lazy
 * module loading the first call on a device may load the library's module
 * and place the array then, so make a first call at set-up time.  All
 * interior cells count (ExcludeBoundCellCalcRes = F, the reference default). */
int paris_calc_residuals_noalloc(int32_t nx, int32_t ny, int32_t nz, int32_t ng, const double* A_dev,
                                 const double* p_dev, double* out3, void* stream);

/* clean_debris, vofmodules.f90:2087-2234 (clean_debris_method, with
 * clean_debris_neighbours <= Ng): 1 sets the interior cells with no cell of
 * the other phase (cvof > 0.5) within `neighbours` cells to their pure phase;
 * 2 sets cells below 0.1 with a neighbourhood sum below 0.3 to 0 and cells
 * above 0.9 within 0.3 of a full neighbourhood to 1; 3 cleans the mixed cells
 * with fewer than 6 mixed cells among their 27 to their phase, in sweeps
 * with the ghosts, flags and clipping refreshed between them (up to 11).
 * Methods 1 and 2 change cvof only, as the reference does; method 3 cvof and
 * vof_flag.  sweeps (may be NULL) gets the number of sweeps run.            */
int paris_clean_debris(paris_handle_t h, int32_t method, int32_t neighbours, int32_t* sweeps);

/* ---- on-disk formats ---------------------------------------------------- */
/* backup_VOF_write, vofmodules.f90:2033-2059: the restart text file of a VOF
 * run (header FORMAT(es17.8e3,7I10) time, itimestep, imin..kmax, then
 * FORMAT(5es25.16e3) u, v, w, p, cvof over k, j, i of the ghosted arrays)
 * from the device fields; an existing file is first renamed <file>.old.   */
int paris_backup_vof_write(paris_handle_t h, const char* filename, double time, int32_t itimestep);
/* backup_VOF_read, vofmodules.f90:2063-2085, and the restart ghosts of
 * paris.f90:3174-3178: loads u, v, w, p, cvof to the device, vof_flag from
 * cvof (get_flags_and_clip), SetVOFBC and the periodic ghosts of cvof, the
 * flags and the velocities.  A file of another grid returns PARIS_BAD_ARGS
 * (the reference stops with "Error: backup_read").  time, itimestep may be
 * NULL.                                                                   */
int paris_backup_vof_read(paris_handle_t h, const char* filename, double* time, int32_t* itimestep);
#define PARIS_VTK_STRUCTURED_GRID    2   /* output_format = 2, output_VOF_VTKSG */
#define PARIS_VTK_STRUCTURED_POINTS  3   /* output_format = 3, output_VOF_VTKSP */
/* output_VOF(nf,i1,i2,j1,j2,k1,k2), vofmodules.f90:1908-2031: one VTK file
 * of cvof over the Fortran index box range = {i1,i2,j1,j2,k1,k2} (1-based,
 * ghosts included: 1..N+2Ng), or NULL for is..ie+1, js..je+1, ks..ke+1 as
 * the step loop writes it; filtered = output_filtered_VOF (27-point filter
 * with weights 8, 4, 2, 1 / 64).                                          */
int paris_output_vof_vtk(paris_handle_t h, const char* filename, int32_t format, double time, const int32_t* range,
                         int32_t filtered);

/* ---- projection adjoint.  No counterpart in the reference: the transpose
 *      of SetupPoisson (modules.f90:2722-2753) + NewSolver + project_velocity
 *      (paris.f90:898-909).  With B_f = 2/(rho_L + rho_R) on every face,
 *      A(B) p = -D u* and u = u* - dt*B*G*p, given gu, gv, gw = dL/du it
 *      returns gus, gvs, gws = dL/du* and gbx, gby, gbz = dL/dB (six face
 *      fields; all nine arrays in the reference layout with ghosts, host or
 *      device memory).  Gradients live on the faces project_velocity updates
 *      (all faces of a periodic direction, the interior faces of a wall-bounded
 *      one); ghost entries of gu/gv/gw are ignored and those of the outputs
 *      are zero (ghost faces are periodic images or boundary constants).
 *      Uses the forward state on the device: RHO, the matrix of the last
 *      paris_setup_poisson (dt must equal its dt) and P as left by the solve.
 *      The transpose solve is the B200 multigrid (A is symmetric); opts as for
 *      paris_new_solver with PARIS_MG_REFERENCE read as PARIS_MG_FP64, or NULL
 *      for FP64 PCG to ||r||/||b|| < 1e-12.  Returns PARIS_NOT_CONVERGED (with
 *      the outputs written) when that tolerance was not reached.  Any output
 *      pointer may be NULL. */
int paris_projection_adjoint(paris_handle_t h, double dt,
                             const double* gu, const double* gv, const double* gw,
                             double* gus, double* gvs, double* gws,
                             double* gbx, double* gby, double* gbz,
                             const paris_solve_opts* opts);

#ifdef __cplusplus
}
#endif
#endif /* PARIS_B200_H */
