"""ctypes view of the C-ABI declared in include/paris_b200.h.

The structures mirror the header field for field; `load_library()` opens the
in-tree shared library built by `build.py` and declares every entry point.
There is no fallback: a missing or unloadable library raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBNAME = "libparis_b200.so"

# status codes
OK, NOT_CONVERGED, NAN_DETECTED, BAD_ARGS, CUDA_ERROR, SETUP_ERROR, NO_DEVICE, CFL_TOO_LARGE = range(8)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "NAN_DETECTED", 3: "BAD_ARGS",
                4: "CUDA_ERROR", 5: "SETUP_ERROR", 6: "NO_DEVICE", 7: "CFL_TOO_LARGE"}

# boundary conditions
BC_WALL, BC_PERIODIC, BC_SHEAR = 0, 1, 2
VOFBC_DRY, VOFBC_WET, VOFBC_JET, VOFBC_PERIODIC, VOFBC_OUTFLOW, VOFBC_90DEG = 0, 1, 2, 3, 4, 5
ADVECT_CIAM, ADVECT_WY = 0, 1
MEAN_ARITH, MEAN_HARM = 101, 102

# fields
(F_CVOF, F_U, F_V, F_W, F_RHO, F_P, F_DU, F_DV, F_DW, F_KAPPA, F_MU, F_VOF_FLAG,
 F_A, F_HEIGHT, F_VOF_PHASE, F_USTAR, F_VSTAR, F_WSTAR, F_MOMENTUM) = range(19)

# solver modes
MG_REFERENCE, MG_FP64, MG_MIXED = 0, 1, 2


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("ng", ctypes.c_int32),
        ("bdry_cond", ctypes.c_int32 * 6),
        ("vofbdry_cond", ctypes.c_int32 * 6),
        ("xlength", ctypes.c_double), ("ylength", ctypes.c_double), ("zlength", ctypes.c_double),
        ("vof_advect", ctypes.c_int32),
        ("dens_mean", ctypes.c_int32),
        ("visc_mean", ctypes.c_int32),
        ("nfilter", ctypes.c_int32),
        ("rho1", ctypes.c_double), ("rho2", ctypes.c_double),
        ("mu1", ctypes.c_double), ("mu2", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("epsc", ctypes.c_double),
        ("nrelax", ctypes.c_int32),
        ("sym_mg", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("mixed_heights", ctypes.c_int32),
        ("use_full_heights", ctypes.c_int32),
        ("do_rotation", ctypes.c_int32),
        ("inject_type", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
        ("jetcenter_yc", ctypes.c_double), ("jetcenter_zc", ctypes.c_double),
        ("radius_liq_inject", ctypes.c_double), ("radius_gas_inject", ctypes.c_double),
    ]


class SolveOpts(ctypes.Structure):
    _fields_ = [
        ("max_error", ctypes.c_double),
        ("rel_tol", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("maxit", ctypes.c_int32),
        ("norm", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("nu1", ctypes.c_int32), ("nu2", ctypes.c_int32),
        ("pcg", ctypes.c_int32),
        ("nu_coarse", ctypes.c_int32), ("coarse_from", ctypes.c_int32), ("coarse_to", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("beta_coarse", ctypes.c_double),
    ]


VTK_STRUCTURED_GRID, VTK_STRUCTURED_POINTS = 2, 3
NSTATS = 25
STATS_RISING_BUBBLE, STATS_PHASE_INVERSION, STATS_TURB = 1, 2, 4


class StatsOpts(ctypes.Structure):
    _fields_ = [
        ("dpdx", ctypes.c_double), ("dpdy", ctypes.c_double), ("dpdz", ctypes.c_double),
        ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
        ("rho_ave", ctypes.c_double),
        ("buoyancy_case", ctypes.c_int32), ("force_valid", ctypes.c_int32), ("test_flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]


def make_stats_opts(dpdx=(0.0, 0.0, 0.0), gravity=(0.0, 0.0, 0.0), rho_ave=0.0, buoyancy=0, force_valid=1,
                    test_flags=0):
    o = StatsOpts()
    o.dpdx, o.dpdy, o.dpdz = (float(a) for a in dpdx)
    o.gx, o.gy, o.gz = (float(a) for a in gravity)
    o.rho_ave, o.buoyancy_case, o.force_valid, o.test_flags = float(rho_ave), int(buoyancy), int(force_valid), \
        int(test_flags)
    return o


class SolveResult(ctypes.Structure):
    _fields_ = [
        ("it", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("res", ctypes.c_double), ("rel_res", ctypes.c_double), ("res0", ctypes.c_double),
    ]


def make_desc(n, length=(1.0, 1.0, 1.0), bc="periodic", vofbc=None, advect=ADVECT_CIAM,
              rho1=1.0, rho2=1.0, mu1=0.0, mu2=0.0, sigma=0.0, epsc=1e-12, nrelax=3,
              sym_mg=0, nfilter=0, dens_mean=MEAN_ARITH, visc_mean=MEAN_ARITH, device=0,
              mixed_heights=1, use_full_heights=1, do_rotation=0, jet=None):
    """Grid descriptor with the reference's namelist defaults.

    bc: "periodic", "wall", or a 6-sequence of BDRY_COND codes (x- y- z- x+ y+ z+).
    vofbc: None (periodic where bc is periodic, 'dry' at walls) or 6 codes.
    jet: None or (inject_type, jetcenter_yc, jetcenter_zc, radius_liq_inject,
    radius_gas_inject) for a 'jet' VOF face.
    """
    d = GridDesc()
    d.nx, d.ny, d.nz = (int(v) for v in n)
    d.ng = 2
    if bc == "periodic":
        bcs = [BC_PERIODIC] * 6
    elif bc == "wall":
        bcs = [BC_WALL] * 6
    else:
        bcs = list(bc)
    if vofbc is None:
        vofbc = [VOFBC_PERIODIC if b == BC_PERIODIC else VOFBC_DRY for b in bcs]
    for i in range(6):
        d.bdry_cond[i] = bcs[i]
        d.vofbdry_cond[i] = vofbc[i]
    d.xlength, d.ylength, d.zlength = (float(v) for v in length)
    d.vof_advect = advect
    d.dens_mean, d.visc_mean, d.nfilter = dens_mean, visc_mean, nfilter
    d.rho1, d.rho2, d.mu1, d.mu2, d.sigma, d.epsc = rho1, rho2, mu1, mu2, sigma, epsc
    d.nrelax, d.sym_mg, d.device = nrelax, sym_mg, device
    d.mixed_heights, d.use_full_heights, d.do_rotation = mixed_heights, use_full_heights, do_rotation
    if jet is not None:
        d.inject_type = int(jet[0])
        d.jetcenter_yc, d.jetcenter_zc, d.radius_liq_inject, d.radius_gas_inject = (float(v) for v in jet[1:5])
    return d


def lib_path():
    return os.path.join(HERE, LIBNAME)


_LIB = None

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int32
CONV_QUICK, CONV_ENO, CONV_SUPERBEE, CONV_WENO = 0, 1, 2, 3

_PROTOS = {
    "paris_gpu_init": (_I, [ctypes.POINTER(GridDesc), ctypes.POINTER(_P)]),
    "paris_gpu_finalize": (_I, [_P]),
    "paris_gpu_upload": (_I, [_P, _I, _P]),
    "paris_gpu_download": (_I, [_P, _I, _P]),
    "paris_gpu_sync": (_I, [_P]),
    "paris_gpu_upload_async": (_I, [_P, _I, _P]),
    "paris_gpu_upload_commit": (_I, [_P, _I]),
    "paris_gpu_download_async": (_I, [_P, _I, _P]),
    "paris_gpu_sync_transfers": (_I, [_P]),
    "paris_gpu_copy_field": (_I, [_P, _I, _I]),
    "paris_gpu_fill_field": (_I, [_P, _I, _D]),
    "paris_gpu_profile": (_I, [_P, _I]),
    "paris_gpu_profile_report": (ctypes.c_int64, [_P, ctypes.c_char_p, ctypes.c_int64]),
    "paris_gpu_stream": (_P, [_P]),
    "paris_gpu_field_ptr": (_P, [_P, _I]),
    "paris_gpu_last_error": (ctypes.c_char_p, [_P]),
    "paris_gpu_launch_count": (ctypes.c_int64, [_P]),
    "paris_vof_sweeps": (_I, [_P, _I, _D]),
    "paris_linfunc": (_I, [_P, _I]),
    "paris_init_spheres": (_I, [_P, _I, _P, _P, _P, _P, _I]),
    "paris_get_all_heights": (_I, [_P]),
    "paris_get_all_curvatures": (_I, [_P, _P]),
    "paris_surface_force": (_I, [_P]),
    "paris_momentum_convection": (_I, [_P, _I]),
    "paris_explicit_mom_diff": (_I, [_P]),
    "paris_volume_force": (_I, [_P, _D, _D, _D, _I, _D, _D, _D, _D]),
    "paris_advance_velocity": (_I, [_P, _D]),
    "paris_set_velocity_bc": (_I, [_P, _P]),
    "paris_time_step_size": (_I, [_P, _D, _D, _D, _P, _P]),
    "paris_get_cfl_and_check": (_I, [_P, _D, _D, _P]),
    "paris_calc_stats": (_I, [_P, ctypes.POINTER(StatsOpts), _P]),
    "paris_clean_debris": (_I, [_P, _I, _I, _P]),
    "paris_vof_mom_sweeps": (_I, [_P, _I, _D, _I, _I, _I, _P]),
    "paris_backup_vof_write": (_I, [_P, ctypes.c_char_p, _D, _I]),
    "paris_backup_vof_read": (_I, [_P, ctypes.c_char_p, _P, _P]),
    "paris_output_vof_vtk": (_I, [_P, ctypes.c_char_p, _I, _D, _P, _I]),
    "paris_setup_poisson": (_I, [_P, _D, _D]),
    "paris_setup_test_mg": (_I, [_P]),
    "paris_new_solver": (_I, [_P, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveResult)]),
    "paris_calc_residuals": (_I, [_P, _P]),
    "paris_mg_test_err": (_I, [_P, _P]),
    "paris_project_velocity": (_I, [_P, _D]),
    "paris_calc_residuals_noalloc": (_I, [_I, _I, _I, _I, _P, _P, _P, _P]),
    "paris_projection_adjoint": (_I, [_P, _D, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                      ctypes.POINTER(SolveOpts)]),
}


def exported_names():
    return list(_PROTOS)


def load_library(path=None):
    """Open the CUDA library; raises OSError when it is missing (no fallback)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or lib_path()
    if not os.path.exists(p):
        raise OSError(f"{p} not built: run __graft_entry__.build() (nvcc, sm_100a)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib
