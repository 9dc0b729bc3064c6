"""The fused sweep with merged phases (one barrier per step) against the
default two-phase form.

Both run the same updates in the same order for every cell; the merged form
runs the second colour of one step and the first colour of the next between
the same two barriers, on 32x12 (PARIS_SWEEP_MERGED=1) or 32x14 (2) tiles,
against 32x16.  A defect-correction solve therefore gives the same pressure
to the bit, a CG solve the same to rounding (its r.z partials come from other
tiles: assert_same_solve).  The environment variable is read when a handle
first builds its FP32 multigrid levels.  Grids: periodic and walled boxes
and mixed boundaries; none of them is a whole number of 12- or 14-row tiles,
so the last tile of every column is partial."""
import os
import warnings

import pytest

from sweep_case import assert_same_solve, problem as _problem

pytestmark = pytest.mark.gpu

KEYS = ("PARIS_SWEEP_MERGED", "PARIS_SWEEP_PAIRS", "PARIS_SWEEP_TMA", "PARIS_SWEEP_RS")


def _solve(runtime, capi, desc, cvof, vel, merged, pcg, opts):
    old = {k: os.environ.get(k) for k in KEYS}
    os.environ["PARIS_SWEEP_MERGED"] = str(merged)
    for k in KEYS[1:]:
        os.environ[k] = "0"
    try:
        with runtime.ParisGpu(desc) as gpu:
            gpu.upload(capi.F_CVOF, cvof)
            for f, a in zip((capi.F_U, capi.F_V, capi.F_W), vel):
                gpu.upload(f, a)
            gpu.linfunc(capi.F_RHO)
            gpu.setup_poisson(1e-3)
            gpu.fill_field(capi.F_P, 0.0)
            r = gpu.new_solver(0.0, maxit=6, mode=capi.MG_MIXED, rel_tol=1e-300, pcg=pcg, **opts)
            return gpu.download(capi.F_P), r
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("opts", [{}, {"beta": 1.1, "beta_coarse": 1.25, "nu_coarse": 4, "coarse_from": 1,
                                       "coarse_to": 2}])
@pytest.mark.parametrize("pcg", [0, 1])
@pytest.mark.parametrize("merged", [1, 2])
@pytest.mark.parametrize("n,bc", [((64, 64, 64), "periodic"), ((64, 64, 64), "wall"),
                                  ((128, 64, 64), (1, 0, 1, 1, 0, 1)), ((64, 128, 64), (0, 1, 0, 0, 1, 0)),
                                  ((128, 128, 128), "periodic")])
def test_merged_sweep_matches_two_phase(gpu_lib, capi, runtime, orc, workloads, n, bc, merged, pcg, opts):
    desc, cvof, vel = _problem(capi, orc, workloads, n, bc, seed=5)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p_m, r_m = _solve(runtime, capi, desc, cvof, vel, merged, pcg, opts)
        p_d, r_d = _solve(runtime, capi, desc, cvof, vel, 0, pcg, opts)
    assert_same_solve(p_m, r_m, p_d, r_d, pcg, True)
