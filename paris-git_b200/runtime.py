"""Host-side mirror of the reference's grid-core subroutines over the C-ABI.

Each method keeps the name and argument meaning of the PARIS subroutine it
replaces (vofsweeps, linfunc, get_all_heights, get_all_curvatures,
surfaceForce, SetupPoisson, NewSolver, project_velocity, calcResiduals,
Setup_testMG, get_MGtest_err).  Arrays are numpy arrays in the reference
layout: float64 (Nz+2Ng, Ny+2Ng, Nx+2Ng) with ghosts, i fastest; A is
(8, Nz, Ny, Nx) = A(is:ie,js:je,ks:ke,8).  Errors raise ParisError; a solver
that reaches maxit returns it = maxit+1 and warns, as NewSolverMG does
(MGsolver.f90:402).
"""
import ctypes
import os
import warnings

import numpy as np

from . import capi


class ParisError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{capi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class ParisGpu:
    """Device-resident grid core for one grid (one CUDA device, no MPI split)."""

    def __init__(self, desc, lib=None):
        self.lib = lib or capi.load_library()
        self.desc = desc
        h = ctypes.c_void_p()
        st = self.lib.paris_gpu_init(ctypes.byref(desc), ctypes.byref(h))
        if st != capi.OK:
            raise ParisError(st, "paris_gpu_init failed")
        self.h = h
        g = desc.ng
        self.shape = (desc.nz + 2 * g, desc.ny + 2 * g, desc.nx + 2 * g)
        self.n = (desc.nx, desc.ny, desc.nz)

    # -- life cycle ---------------------------------------------------------
    def close(self):
        if self.h:
            self.lib.paris_gpu_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != capi.OK:
            err = self.lib.paris_gpu_last_error(self.h)
            raise ParisError(st, f"{what}: {err.decode() if err else ''}")

    # -- transfers ----------------------------------------------------------
    def upload(self, field, arr):
        if field in (capi.F_VOF_FLAG,):
            a = np.ascontiguousarray(arr, dtype=np.int32)
            assert a.shape == self.shape
        elif field == capi.F_A:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            assert a.shape == (8, self.desc.nz, self.desc.ny, self.desc.nx)
        elif field == capi.F_HEIGHT:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            assert a.shape == (6,) + self.shape
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            assert a.shape == self.shape, (a.shape, self.shape)
        self._check(self.lib.paris_gpu_upload(self.h, field, _ptr(a)), "upload")

    def download(self, field):
        if field in (capi.F_VOF_FLAG, capi.F_VOF_PHASE):
            a = np.empty(self.shape, dtype=np.int32)
        elif field == capi.F_A:
            a = np.empty((8, self.desc.nz, self.desc.ny, self.desc.nx))
        elif field == capi.F_HEIGHT:
            a = np.empty((6,) + self.shape)
        else:
            a = np.empty(self.shape)
        self._check(self.lib.paris_gpu_download(self.h, field, _ptr(a)), "download")
        return a

    def download_into(self, field, out):
        """Download a real(8) field into a caller-owned (e.g. pinned) array."""
        assert out.dtype == np.float64 and out.shape == self.shape and out.flags.c_contiguous
        self._check(self.lib.paris_gpu_download(self.h, field, _ptr(out)), "download")

    def upload_from(self, field, arr):
        """Upload without a copy: arr must already be contiguous float64."""
        assert arr.dtype == np.float64 and arr.shape == self.shape and arr.flags.c_contiguous
        self._check(self.lib.paris_gpu_upload(self.h, field, _ptr(arr)), "upload")

    def upload_async(self, field, arr):
        """Start copying a real(8) field to the device (arr: contiguous float64,
        ideally pinned, kept alive and unchanged until sync_transfers); the
        field takes the values at upload_commit."""
        assert arr.dtype == np.float64 and arr.shape == self.shape and arr.flags.c_contiguous
        self._check(self.lib.paris_gpu_upload_async(self.h, field, _ptr(arr)), "upload_async")

    def upload_commit(self, field):
        self._check(self.lib.paris_gpu_upload_commit(self.h, field), "upload_commit")

    def download_async(self, field, out):
        """Asynchronous download into out (contiguous float64, ideally pinned);
        read it only after sync_transfers."""
        assert out.dtype == np.float64 and out.shape == self.shape and out.flags.c_contiguous
        self._check(self.lib.paris_gpu_download_async(self.h, field, _ptr(out)), "download_async")

    def sync_transfers(self):
        self._check(self.lib.paris_gpu_sync_transfers(self.h), "sync_transfers")

    def copy_field(self, dst, src):
        self._check(self.lib.paris_gpu_copy_field(self.h, dst, src), "copy_field")

    def fill_field(self, field, value):
        self._check(self.lib.paris_gpu_fill_field(self.h, field, float(value)), "fill_field")

    def profile(self, enable):
        self._check(self.lib.paris_gpu_profile(self.h, 1 if enable else 0), "profile")

    def profile_report(self):
        """{kernel: (launches, total_ms, cells)} of the events recorded so far."""
        need = self.lib.paris_gpu_profile_report(self.h, None, 0)
        buf = ctypes.create_string_buffer(int(need) + 1)
        self.lib.paris_gpu_profile_report(self.h, buf, len(buf))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms, cells = line.split("\t")
            out[name] = (int(n), float(ms), float(cells))
        return out

    def sync(self):
        self._check(self.lib.paris_gpu_sync(self.h), "sync")

    def stream(self):
        return self.lib.paris_gpu_stream(self.h)

    def field_ptr(self, field):
        return self.lib.paris_gpu_field_ptr(self.h, field)

    def launch_count(self):
        return self.lib.paris_gpu_launch_count(self.h)

    # -- VOF ----------------------------------------------------------------
    def vof_sweeps(self, tswap, dt):
        """vofsweeps(tswap), vofmodules.f90:1340."""
        self._check(self.lib.paris_vof_sweeps(self.h, int(tswap), float(dt)), "vofsweeps")

    vofsweeps = vof_sweeps

    def linfunc(self, which=capi.F_RHO):
        """linfunc(rho,rho1,rho2,DensMean) or (mu,...), vofmodules.f90:171."""
        self._check(self.lib.paris_linfunc(self.h, which), "linfunc")

    def init_spheres(self, centers, radii, refinement=8):
        c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
        r = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).reshape(-1))
        xs = [np.ascontiguousarray(c[:, a]) for a in range(3)]
        self._check(self.lib.paris_init_spheres(self.h, len(r), _ptr(xs[0]), _ptr(xs[1]), _ptr(xs[2]),
                                                _ptr(r), int(refinement)), "init_spheres")

    # -- surface tension ------------------------------------------------------
    def get_all_heights(self):
        self._check(self.lib.paris_get_all_heights(self.h), "get_all_heights")

    def get_all_curvatures(self):
        kappa = np.empty(self.shape)
        self._check(self.lib.paris_get_all_curvatures(self.h, _ptr(kappa)), "get_all_curvatures")
        return kappa

    def surface_force(self):
        self._check(self.lib.paris_surface_force(self.h), "surfaceForce")

    surfaceForce = surface_force

    # -- projection -------------------------------------------------------------
    def setup_poisson(self, dt, volume_source=0.0):
        """SetPressureBC + SetupPoisson(u,v,w,umask,vmask,wmask,rho,dt,A,tmp,VolumeSource)."""
        self._check(self.lib.paris_setup_poisson(self.h, float(dt), float(volume_source)), "SetupPoisson")

    SetupPoisson = setup_poisson

    def setup_test_mg(self):
        self._check(self.lib.paris_setup_test_mg(self.h), "Setup_testMG")

    def new_solver(self, max_error, beta=1.0, maxit=100, norm=2, mode=capi.MG_MIXED, rel_tol=0.0,
                   nu1=2, nu2=2, pcg=0, nu_coarse=0, coarse_from=0, coarse_to=0, beta_coarse=0.0):
        """NewSolver(A,p,maxError,beta,maxit,it,ierr,norm); returns the SolveResult."""
        o = capi.SolveOpts()
        o.max_error, o.rel_tol, o.beta = float(max_error), float(rel_tol), float(beta)
        o.maxit, o.norm, o.mode, o.nu1, o.nu2, o.pcg = int(maxit), int(norm), int(mode), nu1, nu2, int(pcg)
        o.nu_coarse, o.coarse_from, o.coarse_to = int(nu_coarse), int(coarse_from), int(coarse_to)
        o.beta_coarse = float(beta_coarse)
        r = capi.SolveResult()
        st = self.lib.paris_new_solver(self.h, ctypes.byref(o), ctypes.byref(r))
        if st == capi.NOT_CONVERGED:
            warnings.warn(f"Warning: LinearSolver reached maxit: ||res||: {r.res}")
        else:
            self._check(st, "NewSolver")
        return r

    NewSolver = new_solver

    def calc_residuals(self):
        out = np.zeros(3)
        self._check(self.lib.paris_calc_residuals(self.h, _ptr(out)), "calcResiduals")
        return out

    def mg_test_err(self):
        e = ctypes.c_double()
        self._check(self.lib.paris_mg_test_err(self.h, ctypes.byref(e)), "get_MGtest_err")
        return e.value

    def project_velocity(self, dt):
        """project_velocity(), paris.f90:882."""
        self._check(self.lib.paris_project_velocity(self.h, float(dt)), "project_velocity")

    # -- momentum predictor ----------------------------------------------------
    def momentum_convection(self, scheme=capi.CONV_QUICK):
        """momentumConvection(), paris.f90:1957: DU, DV, DW from U, V, W."""
        self._check(self.lib.paris_momentum_convection(self.h, int(scheme)), "momentumConvection")

    def explicit_mom_diff(self):
        """explicitMomDiff(u,v,w,rho,mu,du,dv,dw), paris.f90:2757."""
        self._check(self.lib.paris_explicit_mom_diff(self.h), "explicitMomDiff")

    def volume_force(self, dpdx=0.0, dpdy=0.0, dpdz=0.0, buoyancy=0, gx=0.0, gy=0.0, gz=0.0, rho_ave=0.0):
        """volumeForce(...), paris.f90:2813, with no front-tracking force."""
        self._check(self.lib.paris_volume_force(self.h, float(dpdx), float(dpdy), float(dpdz), int(buoyancy),
                                                float(gx), float(gy), float(gz), float(rho_ave)), "volumeForce")

    def advance_velocity(self, dt):
        """u = u + dt*du, paris.f90:442."""
        self._check(self.lib.paris_advance_velocity(self.h, float(dt)), "advance_velocity")

    def set_velocity_bc(self, wall_vel=None):
        """SetVelocityBC for walls / periodic boundaries + do_ghost_vector.
        wall_vel: WallVel as a (6, 3) array (face, component) or None."""
        if wall_vel is None:
            self._check(self.lib.paris_set_velocity_bc(self.h, None), "SetVelocityBC")
        else:
            wv = np.ascontiguousarray(np.asarray(wall_vel, dtype=np.float64).reshape(6, 3).T)   # Fortran order
            self._check(self.lib.paris_set_velocity_bc(self.h, _ptr(wv)), "SetVelocityBC")

    def vof_mom_sweeps(self, tswap, dt, staggered=True, lin_interp=False, scheme=capi.CONV_QUICK, wall_vel=None):
        """vofandmomsweepsstaggered (DoMOMCONS): the momentum of each component
        advected with the split VOF fluxes of its control volume; DU/DV/DW
        replaced where the advected fraction is mixed.  The MOMENTUM field
        is kept between calls."""
        wv = None if wall_vel is None else np.ascontiguousarray(
            np.asarray(wall_vel, dtype=np.float64).reshape(6, 3).T)
        self._check(self.lib.paris_vof_mom_sweeps(self.h, int(tswap), float(dt), 1 if staggered else 0,
                                                  1 if lin_interp else 0, int(scheme), _ptr(wv) if wv is not None
                                                  else None), "vofandmomsweepsstaggered")

    # -- time-step control and statistics ------------------------------------
    def time_step_size(self, cfl, max_dt, u_inject=0.0):
        """TimeStepSize (no free surface): returns (dt, vmax)."""
        dt, vmax = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.paris_time_step_size(self.h, float(cfl), float(max_dt), float(u_inject),
                                                  ctypes.byref(dt), ctypes.byref(vmax)), "TimeStepSize")
        return dt.value, vmax.value

    def get_cfl_and_check(self, dt, cflmax_allowed=0.5):
        """get_cfl_and_check: returns the CFL number; raises ParisError
        (CFL_TOO_LARGE) above cflmax_allowed, where the reference stops."""
        cfl = ctypes.c_double()
        self._check(self.lib.paris_get_cfl_and_check(self.h, float(dt), float(cflmax_allowed), ctypes.byref(cfl)),
                    "get_cfl_and_check")
        return cfl.value

    def calc_stats(self, opts=None, **kw):
        """calcStats: the 25 columns stats(1:25) as a float64 array.  opts: a
        capi.StatsOpts, or keyword arguments of capi.make_stats_opts."""
        o = opts if opts is not None else capi.make_stats_opts(**kw)
        out = np.zeros(capi.NSTATS)
        self._check(self.lib.paris_calc_stats(self.h, ctypes.byref(o), _ptr(out)), "calcStats")
        return out

    calcStats = calc_stats

    def clean_debris(self, method=1, neighbours=2):
        """clean_debris (clean_debris_method, clean_debris_neighbours);
        returns the number of sweeps run."""
        n = ctypes.c_int32()
        self._check(self.lib.paris_clean_debris(self.h, int(method), int(neighbours), ctypes.byref(n)),
                    "clean_debris")
        return n.value

    # -- on-disk formats --------------------------------------------------------
    def backup_vof_write(self, filename, time, itimestep):
        """backup_VOF_write: the restart text file from the device fields."""
        self._check(self.lib.paris_backup_vof_write(self.h, os.fsencode(filename), float(time), int(itimestep)),
                    "backup_VOF_write")

    def backup_vof_read(self, filename):
        """backup_VOF_read (+ the restart ghosts): returns (time, itimestep)."""
        t, it = ctypes.c_double(), ctypes.c_int32()
        self._check(self.lib.paris_backup_vof_read(self.h, os.fsencode(filename), ctypes.byref(t), ctypes.byref(it)),
                    "backup_VOF_read")
        return t.value, it.value

    def output_vof_vtk(self, filename, fmt=capi.VTK_STRUCTURED_GRID, time=0.0, index_range=None, filtered=False):
        """output_VOF: one VTK file of cvof; index_range = (i1, i2, j1, j2,
        k1, k2) in Fortran indices or None for is..ie+1 etc."""
        rng = None if index_range is None else (ctypes.c_int32 * 6)(*[int(v) for v in index_range])
        self._check(self.lib.paris_output_vof_vtk(self.h, os.fsencode(filename), int(fmt), float(time), rng,
                                                  1 if filtered else 0), "output_VOF")

    def ns_step(self, itimestep, dt, scheme=capi.CONV_QUICK, gravity=(0.0, 0.0, 0.0), buoyancy=0, rho_ave=0.0,
                dpdx=(0.0, 0.0, 0.0), wall_vel=None, solve=None, clean_debris=None, momcons=None):
        """One explicit time step in the order of the PARIS step loop
        (paris.f90:281-656: itime_scheme 1, two-phase VOF, no front
        tracking, no free surface): property update, momentum convection,
        VOF sweeps, heights, density, surface tension (when sigma > 0),
        viscous diffusion, volume force, u += dt*du, velocity BCs, then the
        projection (SetupPoisson, NewSolver, project_velocity, velocity BCs)
        and the property update.  `solve`: keyword arguments of new_solver
        (default: the B200 mixed solver to ||r||/||b|| < 1e-10).
        clean_debris: (method, neighbours, nsteps) to run clean_debris after
        the VOF sweeps of every nsteps-th step (do_clean_debris), or None.
        momcons: None, or the keyword arguments staggered / lin_interp of
        vof_mom_sweeps, run before the VOF sweeps (DoMOMCONS).
        Returns the solver's result."""
        solve = dict(solve or {"max_error": 0.0, "rel_tol": 1e-10, "maxit": 200, "mode": capi.MG_MIXED, "pcg": 1})
        for f in (capi.F_DU, capi.F_DV, capi.F_DW):
            self.fill_field(f, 0.0)
        self.linfunc(capi.F_RHO)
        self.linfunc(capi.F_MU)
        self.momentum_convection(scheme)
        if momcons is not None:
            self.vof_mom_sweeps(itimestep, dt, scheme=scheme, wall_vel=wall_vel, **momcons)
        self.vof_sweeps(itimestep, dt)
        if clean_debris is not None and itimestep % clean_debris[2] == 0:
            self.clean_debris(clean_debris[0], clean_debris[1])
        self.get_all_heights()
        self.linfunc(capi.F_RHO)
        if self.desc.sigma > 0.0:
            self.surface_force()
        self.explicit_mom_diff()
        self.volume_force(dpdx[0], dpdx[1], dpdx[2], buoyancy, gravity[0], gravity[1], gravity[2], rho_ave)
        self.advance_velocity(dt)
        self.set_velocity_bc(wall_vel)
        self.setup_poisson(dt)
        r = self.new_solver(**solve)
        self.project_velocity(dt)
        self.set_velocity_bc(wall_vel)
        self.linfunc(capi.F_RHO)
        self.linfunc(capi.F_MU)
        return r

    def projection_adjoint(self, dt, g, rel_tol=1e-12, maxit=100, mode=capi.MG_FP64, pcg=1):
        """Reverse mode of setup_poisson + new_solver + project_velocity.

        g: dL/du, dL/dv, dL/dw (layout-shaped float64 arrays).  Returns
        ([dL/du*, dL/dv*, dL/dw*], [dL/dBx, dL/dBy, dL/dBz]) with
        B = 2/(rho_L + rho_R) the face coefficient; the forward state (RHO,
        the SetupPoisson matrix, P) must still be on the device."""
        o = capi.SolveOpts()
        o.max_error, o.rel_tol, o.beta = 0.0, float(rel_tol), 1.0
        o.maxit, o.norm, o.mode, o.nu1, o.nu2, o.pcg = int(maxit), 2, int(mode), 2, 2, int(pcg)
        gg = [np.ascontiguousarray(a, dtype=np.float64) for a in g]
        for a in gg:
            if a.shape != self.shape:
                raise ValueError("projection_adjoint: gradient arrays must have the layout's shape")
        gs = [np.empty(self.shape) for _ in range(3)]
        gb = [np.empty(self.shape) for _ in range(3)]
        st = self.lib.paris_projection_adjoint(self.h, float(dt), *(_ptr(a) for a in gg), *(_ptr(a) for a in gs),
                                               *(_ptr(a) for a in gb), ctypes.byref(o))
        if st == capi.NOT_CONVERGED:
            warnings.warn("projection_adjoint: transpose solve did not reach the tolerance")
        else:
            self._check(st, "projection_adjoint")
        return gs, gb
