"""ctypes binding of the CPU oracle (liboracle.so).

Test infrastructure only: the parity checker used by tests/, by
__graft_entry__.smoke() and by the cpu_baseline leg of bench.py.  Arrays are
numpy float64/int32 arrays of shape (Nzt, Nyt, Nxt) (= Fortran
(imin:imax,jmin:jmax,kmin:kmax), i fastest), the matrix A has shape
(8, nz, ny, nx) (= A(is:ie,js:je,ks:ke,8)).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def _grid_desc_type():
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    return pkg.capi


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        D = ctypes.c_double
        I = ctypes.c_int
        capi = _grid_desc_type()
        G = ctypes.POINTER(capi.GridDesc)
        protos = {
            "og_setup_poisson": (I, [G, P, P, P, P, D, D, P]),
            "og_setup_testmg": (I, [G, P, P]),
            "og_new_solver_mg": (I, [G, P, P, D, D, I, I, P, P, P]),
            "og_new_solver_mg_timed": (I, [G, P, P, D, D, I, I, P, P, P, D]),
            "og_calc_residual": (D, [G, P, P, I]),
            "og_mgtest_err": (D, [G, P]),
            "og_project_velocity": (I, [G, P, P, P, P, P, D]),
            "og_fill_ghosts": (None, [G, P]),
            "og_vofsweeps": (I, [G, I, D, P, P, P, P, P, P]),
            "og_flags_clip": (I, [G, P, P]),
            "og_setvofbc_host": (I, [G, P, P]),
            "og_linfunc": (I, [G, P, P, D, D, I]),
            "og_init_spheres": (I, [G, I, P, P, P, P, I, I, P, P, P]),
            "og_fastmg_solve": (I, [G, P, P, D, I, I, I, I, I, D, D, I, I, I, P]),
            "og_get_all_heights": (I, [G, P, P, P]),
            "og_get_all_curvatures": (I, [G, P, P, P, P, P, P]),
            "og_surface_force": (I, [G, P, P, P, P, P, P]),
            "og_al3d": (D, [P, D]),
            "og_cc3d": (D, [P, D]),
            "og_fl3d": (D, [P, D, P, P]),
            "og_area3d": (D, [P, D]),
            "og_area_centroid": (None, [P, D, P]),
            "og_mycs": (None, [P, P]),
            "og_fd32": (None, [P, P]),
            "og_face_B": (None, [G, P, P, P, P]),
            "og_momentum_convection": (I, [G, I, P, P, P, P, P, P]),
            "og_explicit_mom_diff": (I, [G, P, P, P, P, P, P, P, P]),
            "og_volume_force": (I, [G, P, D, D, D, I, D, D, D, D, P, P, P]),
            "og_advance_velocity": (I, [G, D, P, P, P, P, P, P]),
            "og_set_velocity_bc": (I, [G, P, P, P, P]),
            "og_projection_forward_B": (I, [G, D, P, P, P, P, P, P, P, P, P, P, D, I]),
            "og_projection_adjoint": (I, [G, D, P, P, P, P, P, P, P, P, P, P, P, P, P, D, I]),
            "og_time_step_size": (I, [G, P, P, P, D, D, D, P, P]),
            "og_clean_debris": (I, [G, P, P, I, I, P]),
            "og_vof_mom_sweeps": (I, [G, I, D, I, I, I, P, P, P, P, P, P, P, P, P, P]),
            "og_init_shapes": (I, [G, I, P, P, P, P, P, I, I, P, P, P]),
            "og_init_wave": (I, [G, I, I, D, I, P, P, P]),
            "og_flux_centroid": (None, [P, D, P, P, P]),
            "og_get_cfl_and_check": (I, [G, P, P, P, D, D, P]),
            "og_calc_stats": (I, [G, P, P, P, P, P, P, P, P, ctypes.POINTER(capi.StatsOpts), P, P]),
        }
        for name, (res, args) in protos.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def shape(desc):
    return (desc.nz + 2 * desc.ng, desc.ny + 2 * desc.ng, desc.nx + 2 * desc.ng)


def zeros(desc, dtype=np.float64):
    return np.zeros(shape(desc), dtype=dtype)


def interior(desc, a):
    g = desc.ng
    return a[g:g + desc.nz, g:g + desc.ny, g:g + desc.nx]


def fill_ghosts(desc, F):
    lib().og_fill_ghosts(ctypes.byref(desc), _p(F))


def setup_poisson(desc, u, v, w, rho, dt, volsrc=0.0):
    A = np.zeros((8, desc.nz, desc.ny, desc.nx))
    st = lib().og_setup_poisson(ctypes.byref(desc), _p(u), _p(v), _p(w), _p(rho), dt, volsrc, _p(A))
    return st, A


def setup_testmg(desc, rho):
    A = np.zeros((8, desc.nz, desc.ny, desc.nx))
    lib().og_setup_testmg(ctypes.byref(desc), _p(rho), _p(A))
    return A


def new_solver_mg(desc, A, p, max_error, beta=1.0, maxit=20, norm=2):
    """NewSolverMG on (A, p); p updated in place. Returns (status, it, tres2, history)."""
    it = ctypes.c_int(0)
    t = ctypes.c_double(0)
    hist = np.zeros(max(maxit, 1))
    st = lib().og_new_solver_mg(ctypes.byref(desc), _p(np.ascontiguousarray(A)), _p(p), max_error,
                                beta, maxit, norm, ctypes.byref(it), ctypes.byref(t), _p(hist))
    return st, it.value, t.value, hist[:min(it.value, maxit)]


def new_solver_mg_timed(desc, A, p, max_error, max_seconds, beta=1.0, maxit=100000, norm=2):
    """NewSolverMG that also stops after the first V-cycle ending past
    max_seconds.  Returns (converged, cycles, tres2, history)."""
    it = ctypes.c_int(0)
    t = ctypes.c_double(0)
    hist = np.zeros(max(maxit, 1))
    st = lib().og_new_solver_mg_timed(ctypes.byref(desc), _p(np.ascontiguousarray(A)), _p(p), max_error, beta,
                                      maxit, norm, ctypes.byref(it), ctypes.byref(t), _p(hist), float(max_seconds))
    n = min(it.value, maxit)
    return st == 0, n, t.value, hist[:n]


def calc_residual(desc, A, p, normorder):
    return lib().og_calc_residual(ctypes.byref(desc), _p(A), _p(p), normorder)


def mgtest_err(desc, p):
    return lib().og_mgtest_err(ctypes.byref(desc), _p(p))


def project_velocity(desc, u, v, w, p, rho, dt):
    return lib().og_project_velocity(ctypes.byref(desc), _p(u), _p(v), _p(w), _p(p), _p(rho), dt)


def vofsweeps(desc, tswap, dt, cvof, flag, u, v, w, phase=None):
    return lib().og_vofsweeps(ctypes.byref(desc), tswap, dt, _p(cvof), _p(flag), _p(phase),
                              _p(u), _p(v), _p(w))


def flags_clip(desc, c, f):
    return lib().og_flags_clip(ctypes.byref(desc), _p(c), _p(f))


def setvofbc(desc, cvof, flag):
    """SetVOFBC(cvof, vof_flag) in place (vofmodules.f90:1694-1825)."""
    return lib().og_setvofbc_host(ctypes.byref(desc), _p(cvof), _p(flag))


def linfunc(desc, cvof, a1, a2, meanflag):
    field = zeros(desc)
    lib().og_linfunc(ctypes.byref(desc), _p(field), _p(cvof), a1, a2, meanflag)
    return field


def init_shapes(desc, centers, radii, excentricity=(0.0, 0.0, 0.0), ipar=0, refinement=8):
    """levelset2vof(shapes2ls, ipar): spheres (ipar 0) or one cylinder along
    x/y/z (ipar -1/-2/-3), with the excentricity of the bubbles."""
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    r = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).reshape(-1))
    xc, yc, zc = (np.ascontiguousarray(c[:, a]) for a in range(3))
    e = np.ascontiguousarray(np.asarray(excentricity, dtype=np.float64))
    cvof = zeros(desc)
    flag = zeros(desc, np.int32)
    phase = zeros(desc, np.int32)
    st = lib().og_init_shapes(ctypes.byref(desc), len(r), _p(xc), _p(yc), _p(zc), _p(r), _p(e), ipar, refinement,
                              _p(cvof), _p(flag), _p(phase))
    assert st == 0, st
    return cvof, flag, phase


def init_wave(desc, ipar=3, normal_up=True, hshift=0.0, refinement=8):
    """levelset2vof(wave2ls, ipar): the cosine interface of the height and
    capillary-wave tests (amplitude one cell, A_h = 2)."""
    cvof = zeros(desc)
    flag = zeros(desc, np.int32)
    phase = zeros(desc, np.int32)
    st = lib().og_init_wave(ctypes.byref(desc), ipar, 1 if normal_up else 0, hshift, refinement, _p(cvof), _p(flag),
                            _p(phase))
    assert st == 0, st
    return cvof, flag, phase


def init_spheres(desc, centers, radii, refinement=8, jacobi=False):
    """levelset2vof(shapes2ls): jacobi=False is the reference's in-place loop
    order; True reads pass-1 flags only (the device's order-free variant)."""
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    r = np.ascontiguousarray(np.asarray(radii, dtype=np.float64).reshape(-1))
    xc, yc, zc = (np.ascontiguousarray(c[:, a]) for a in range(3))
    cvof = zeros(desc)
    flag = zeros(desc, np.int32)
    phase = zeros(desc, np.int32)
    st = lib().og_init_spheres(ctypes.byref(desc), len(r), _p(xc), _p(yc), _p(zc), _p(r), refinement,
                               1 if jacobi else 0, _p(cvof), _p(flag), _p(phase))
    if st:
        raise ValueError("ls2vof_refined: bad flag (largest vof_flag after the first pass is not 2)")
    return cvof, flag, phase


def _v3(n):
    return np.ascontiguousarray(np.asarray(n, dtype=np.float64).reshape(3))


def al3d(n, c):
    return lib().og_al3d(_p(_v3(n)), c)


def cc3d(n, alpha):
    return lib().og_cc3d(_p(_v3(n)), alpha)


def fl3d(n, alpha, x0, dx):
    return lib().og_fl3d(_p(_v3(n)), alpha, _p(_v3(x0)), _p(_v3(dx)))


def area3d(n, c):
    return lib().og_area3d(_p(_v3(n)), c)


def area_centroid(n, c):
    out = np.zeros(3)
    lib().og_area_centroid(_p(_v3(n)), c, _p(out))
    return out


def mycs(block):
    """block: 3x3x3 array indexed [i,j,k] (Fortran c(0:2,0:2,0:2))."""
    b = np.ascontiguousarray(np.asarray(block, dtype=np.float64).transpose(2, 1, 0))
    out = np.zeros(3)
    lib().og_mycs(_p(b), _p(out))
    return out


def grid_coords(desc):
    """x, xh, dx, dxh (and y, z) of paris.f90:3057-3100, index = Fortran-1."""
    out = {}
    for ax, n, L in (("x", desc.nx, desc.xlength), ("y", desc.ny, desc.ylength), ("z", desc.nz, desc.zlength)):
        ng = desc.ng
        nt = n + 2 * ng
        xh = np.array([L * (0.0 * s * (0.5 - s) * (1.0 - s) + s) for s in ((f - ng) / n for f in range(1, nt + 1))])
        x = np.zeros(nt)
        x[1:] = 0.5 * (xh[1:] + xh[:-1])
        x[0] = 2.0 * xh[0] - x[1]
        out[ax] = x
        out[ax + "h"] = xh
    return out


def fastmg_solve(desc, A, p_int, rel_tol, maxit=100, mixed=True, pcg=False, nu1=2, nu2=2, omega=1.0,
                 nu_coarse=0, coarse_from=0, coarse_to=0, omega_coarse=0.0):
    """The B200 solver's own MG restated on the CPU; p_int: interior (nz,ny,nx);
    omega: relaxation factor of the red-black smoother (omega_coarse > 0: the
    factor on the levels below the finest); nu_coarse sweeps each way on the
    levels coarse_from (0: 1) .. coarse_to (0: the coarsest) when
    nu_coarse > 0."""
    hist = np.zeros(maxit)
    p = np.ascontiguousarray(p_int, dtype=np.float64)
    it = lib().og_fastmg_solve(ctypes.byref(desc), _p(np.ascontiguousarray(A)), _p(p), rel_tol, maxit,
                               1 if mixed else 0, 1 if pcg else 0, nu1, nu2, float(omega), float(omega_coarse),
                               int(nu_coarse), int(coarse_from), int(coarse_to), _p(hist))
    return p, it, hist[:it]


def get_all_heights(desc, cvof, flag):
    """get_all_heights: returns height (6, Nzt, Nyt, Nxt)."""
    H = np.zeros((6,) + shape(desc))
    lib().og_get_all_heights(ctypes.byref(desc), _p(np.ascontiguousarray(cvof)),
                             _p(np.ascontiguousarray(flag, dtype=np.int32)), _p(H))
    return H


def get_all_curvatures(desc, cvof, flag, H):
    """get_all_curvatures: returns (kappa, kappaflag, method_count)."""
    kap = zeros(desc)
    kf = zeros(desc, np.int32)
    mc = np.zeros(5, dtype=np.int32)
    lib().og_get_all_curvatures(ctypes.byref(desc), _p(np.ascontiguousarray(cvof)),
                                _p(np.ascontiguousarray(flag, dtype=np.int32)), _p(np.ascontiguousarray(H)),
                                _p(kap), _p(kf), _p(mc))
    return kap, kf, mc


def surface_force(desc, cvof, kappa, rho, du, dv, dw):
    return lib().og_surface_force(ctypes.byref(desc), _p(cvof), _p(kappa), _p(rho), _p(du), _p(dv), _p(dw))


def face_B(desc, rho):
    """B_f = 2/(rho_L + rho_R) on the faces project_velocity updates."""
    B = [zeros(desc) for _ in range(3)]
    lib().og_face_B(ctypes.byref(desc), _p(np.ascontiguousarray(rho)), *(_p(b) for b in B))
    return B


def projection_forward_B(desc, dt, B, ustar, rel_tol=1e-15, maxit=60):
    """SetupPoisson + solve + project_velocity with the face coefficients B
    as the parameters.  Returns ([u, v, w], p, cycles)."""
    us = [np.ascontiguousarray(a, dtype=np.float64) for a in ustar]
    out = [zeros(desc) for _ in range(3)]
    p = zeros(desc)
    it = lib().og_projection_forward_B(ctypes.byref(desc), dt, *(_p(np.ascontiguousarray(b)) for b in B),
                                       *(_p(a) for a in us), *(_p(a) for a in out), _p(p), rel_tol, maxit)
    return out, p, it


def projection_adjoint(desc, dt, B, p, g, rel_tol=1e-15, maxit=60):
    """dL/du* and dL/dB of the projection given g = dL/du.  Returns
    ([gu*, gv*, gw*], [gBx, gBy, gBz], cycles)."""
    gs = [zeros(desc) for _ in range(3)]
    gb = [zeros(desc) for _ in range(3)]
    gg = [np.ascontiguousarray(a, dtype=np.float64) for a in g]
    it = lib().og_projection_adjoint(ctypes.byref(desc), dt, *(_p(np.ascontiguousarray(b)) for b in B),
                                     _p(np.ascontiguousarray(p)), *(_p(a) for a in gg), *(_p(a) for a in gs),
                                     *(_p(a) for a in gb), rel_tol, maxit)
    return gs, gb, it


def updated_faces(desc, d):
    """Boolean mask (layout shape) of the faces of direction d (0=x) that
    project_velocity updates."""
    m = np.zeros(shape(desc), dtype=bool)
    g = desc.ng
    n = (desc.nx, desc.ny, desc.nz)
    per = desc.bdry_cond[d] == 1
    hi = [n[0], n[1], n[2]]
    if not per:
        hi[d] -= 1
    m[g:g + hi[2], g:g + hi[1], g:g + hi[0]] = True
    return m


def momentum_convection(desc, scheme, u, v, w, du, dv, dw):
    """momentumConvection: assigns du, dv, dw (in place) from u, v, w."""
    return lib().og_momentum_convection(ctypes.byref(desc), scheme, _p(u), _p(v), _p(w), _p(du), _p(dv), _p(dw))


def explicit_mom_diff(desc, u, v, w, rho, mu, du, dv, dw):
    return lib().og_explicit_mom_diff(ctypes.byref(desc), _p(u), _p(v), _p(w), _p(rho), _p(mu), _p(du), _p(dv),
                                      _p(dw))


def volume_force(desc, rho, du, dv, dw, dpdx=0.0, dpdy=0.0, dpdz=0.0, buoyancy=0, gx=0.0, gy=0.0, gz=0.0,
                 rho_ave=0.0):
    return lib().og_volume_force(ctypes.byref(desc), _p(rho), dpdx, dpdy, dpdz, buoyancy, gx, gy, gz, rho_ave,
                                 _p(du), _p(dv), _p(dw))


def advance_velocity(desc, dt, u, v, w, du, dv, dw):
    return lib().og_advance_velocity(ctypes.byref(desc), dt, _p(u), _p(v), _p(w), _p(du), _p(dv), _p(dw))


def set_velocity_bc(desc, u, v, w, wall_vel=None):
    """wall_vel: (6, 3) array WallVel(face, component) or None."""
    wv = None if wall_vel is None else np.ascontiguousarray(np.asarray(wall_vel, dtype=np.float64).reshape(6, 3).T)
    return lib().og_set_velocity_bc(ctypes.byref(desc), _p(u), _p(v), _p(w), _p(wv))


def vof_mom_sweeps(desc, tswap, dt, cvof, flag, u, v, w, du, dv, dw, mom, staggered=True, lin_interp=False,
                   scheme=0, wall_vel=None):
    """vofandmomsweepsstaggered (DoMOMCONS): advects the momentum of each
    component with the split VOF fluxes and overwrites du, dv, dw where the
    advected (staggered) fraction is mixed; mom is the persistent momentum
    array (in/out).  cvof and flag are read only."""
    wv = None if wall_vel is None else np.ascontiguousarray(np.asarray(wall_vel, dtype=np.float64).reshape(6, 3).T)
    f32 = np.ascontiguousarray(flag, dtype=np.int32)
    st = lib().og_vof_mom_sweeps(ctypes.byref(desc), tswap, dt, 1 if staggered else 0, 1 if lin_interp else 0, scheme,
                                 _p(wv), _p(cvof), _p(f32), _p(u), _p(v), _p(w), _p(du), _p(dv), _p(dw), _p(mom))
    assert st == 0, st


def flux_centroid(nr, alpha, x0, dx):
    out = np.zeros(3)
    lib().og_flux_centroid(_p(np.ascontiguousarray(nr, dtype=np.float64)), alpha,
                           _p(np.ascontiguousarray(x0, dtype=np.float64)),
                           _p(np.ascontiguousarray(dx, dtype=np.float64)), _p(out))
    return out


def ns_step(desc, st, itimestep, dt, scheme=0, gravity=(0.0, 0.0, 0.0), buoyancy=0, rho_ave=0.0,
            dpdx=(0.0, 0.0, 0.0), wall_vel=None, max_error=1e-12, maxit=2000, rel_tol=None, clean_debris=None,
            momcons=None, solver="mg_ref"):
    """The step loop of paris.f90:281-656 (explicit, two-phase VOF, no front
    tracking, no free surface) on the oracle; st: dict of ghosted arrays
    cvof, flag, u, v, w, p, rho, mu (updated in place).  The pressure is
    solved by the reference multigrid to the absolute RMS residual
    max_error, or, with rel_tol, to rel_tol times the RMS of the right-hand
    side (||r||_2/||b||_2 < rel_tol).  momcons: None, or the keyword
    arguments staggered / lin_interp of vof_mom_sweeps to run the
    momentum-conserving sweeps before vofsweeps (DoMOMCONS, paris.f90:303-305);
    st["mom"] then holds the persistent momentum array.  solver: "mg_ref"
    (NewSolverMG, power-of-two grids) or "fast" (the FP64 restatement of the
    B200 solver, FCG preconditioned by V(2,2) cycles, to rel_tol; any even
    grid).  Returns the solver's iteration count."""
    u, v, w = st["u"], st["v"], st["w"]
    du, dv, dw = (zeros(desc) for _ in range(3))
    rho = linfunc(desc, st["cvof"], desc.rho1, desc.rho2, desc.dens_mean)
    mu = linfunc(desc, st["cvof"], desc.mu1, desc.mu2, desc.visc_mean)
    momentum_convection(desc, scheme, u, v, w, du, dv, dw)
    if momcons is not None:
        if "mom" not in st:
            st["mom"] = zeros(desc)
        vof_mom_sweeps(desc, itimestep, dt, st["cvof"], st["flag"], u, v, w, du, dv, dw, st["mom"], scheme=scheme,
                       wall_vel=wall_vel, **momcons)
    vofsweeps(desc, itimestep, dt, st["cvof"], st["flag"], u, v, w)
    if clean_debris is not None and itimestep % clean_debris[2] == 0:   # paris.f90:310-314
        globals()["clean_debris"](desc, st["cvof"], st["flag"], clean_debris[0], clean_debris[1])
    H = get_all_heights(desc, st["cvof"], st["flag"])
    rho = linfunc(desc, st["cvof"], desc.rho1, desc.rho2, desc.dens_mean)
    if desc.sigma > 0.0:
        kap, _, _ = get_all_curvatures(desc, st["cvof"], st["flag"], H)
        surface_force(desc, st["cvof"], kap, rho, du, dv, dw)
    explicit_mom_diff(desc, u, v, w, rho, mu, du, dv, dw)
    volume_force(desc, rho, du, dv, dw, dpdx[0], dpdx[1], dpdx[2], buoyancy, gravity[0], gravity[1], gravity[2],
                 rho_ave)
    advance_velocity(desc, dt, u, v, w, du, dv, dw)
    set_velocity_bc(desc, u, v, w, wall_vel)
    _, A = setup_poisson(desc, u, v, w, rho, dt)
    if solver == "fast":
        # an absolute max_error (the reference's MAXERROR) becomes the relative
        # tolerance it stands for; a right-hand side already below it needs no solve
        rms = float(np.sqrt(np.mean(A[7] ** 2)))
        tol = rel_tol if rel_tol is not None else (max_error / rms if rms > 0.0 else 1.0)
        it = 0
        if tol < 1.0:
            p_int, it, _ = fastmg_solve(desc, A, np.ascontiguousarray(interior(desc, st["p"])), tol, maxit=maxit,
                                        mixed=False, pcg=True)
            interior(desc, st["p"])[...] = p_int
            fill_ghosts(desc, st["p"])
    else:
        if rel_tol is not None:
            max_error = rel_tol * float(np.sqrt(np.mean(A[7] ** 2)))
        status, it, _, _ = new_solver_mg(desc, A, st["p"], max_error, maxit=maxit)
        assert status in (0, 1), status   # OK or not converged; anything else is a refused grid
    project_velocity(desc, u, v, w, st["p"], rho, dt)
    set_velocity_bc(desc, u, v, w, wall_vel)
    st["rho"] = linfunc(desc, st["cvof"], desc.rho1, desc.rho2, desc.dens_mean)
    st["mu"] = linfunc(desc, st["cvof"], desc.mu1, desc.mu2, desc.visc_mean)
    return it


def time_step_size(desc, u, v, w, cfl, max_dt, u_inject=0.0):
    """TimeStepSize (no free surface): returns (dt, vmax)."""
    dt, vmax = ctypes.c_double(), ctypes.c_double()
    st = lib().og_time_step_size(ctypes.byref(desc), _p(u), _p(v), _p(w), cfl, max_dt, u_inject, ctypes.byref(dt),
                                 ctypes.byref(vmax))
    assert st == 0
    return dt.value, vmax.value


def get_cfl_and_check(desc, u, v, w, dt, cflmax_allowed=0.5):
    """get_cfl_and_check: returns (status, cfl)."""
    cfl = ctypes.c_double()
    st = lib().og_get_cfl_and_check(ctypes.byref(desc), _p(u), _p(v), _p(w), dt, cflmax_allowed, ctypes.byref(cfl))
    return st, cfl.value


def calc_stats(desc, u, v, w, rho, p, cvof, mu, flag, opts=None):
    """calcStats: returns (stats(1:25), sums of |term| per column)."""
    capi = _grid_desc_type()
    out, ab = np.zeros(25), np.zeros(25)
    f32 = np.ascontiguousarray(flag, dtype=np.int32)
    st = lib().og_calc_stats(ctypes.byref(desc), _p(u), _p(v), _p(w), _p(rho), _p(p), _p(cvof), _p(mu), _p(f32),
                             ctypes.byref(opts) if opts is not None else None, _p(out), _p(ab))
    assert st == 0, st
    return out, ab


def clean_debris(desc, cvof, flag, method=1, neighbours=2):
    """clean_debris on cvof (float64) and flag (int32) in place; returns the sweeps run."""
    assert cvof.dtype == np.float64 and flag.dtype == np.int32
    n = ctypes.c_int()
    st = lib().og_clean_debris(ctypes.byref(desc), _p(cvof), _p(flag), method, neighbours, ctypes.byref(n))
    assert st == 0, st
    return n.value
