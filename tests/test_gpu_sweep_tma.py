"""The TMA-staged fused sweep against the cp.async-staged one.

The two kernels share the tiles, the wavefront and the arithmetic of the
fused red-black sweep and differ only in how the planes reach shared memory,
so a defect-correction solve with either gives the same pressure to the bit
(a CG solve the same to rounding: assert_same_solve).  The
environment variable PARIS_SWEEP_TMA, read when a handle first builds its
FP32 multigrid levels, selects the TMA staging (1) or the cp.async one (0,
the default); both arms run the sweeps one at a time (PARIS_SWEEP_PAIRS=0).
Grids: periodic and walled boxes, and mixed boundaries, whose fused levels
(at least 32^3 cells) have the first and last tiles of every row and column
wrapped or zero."""
import os

import numpy as np
import pytest

from sweep_case import assert_same_solve, problem as _problem

pytestmark = pytest.mark.gpu


def _solve(runtime, capi, desc, cvof, vel, tma, pcg):
    old = {k: os.environ.get(k) for k in ("PARIS_SWEEP_TMA", "PARIS_SWEEP_PAIRS")}
    os.environ["PARIS_SWEEP_TMA"] = "1" if tma else "0"
    os.environ["PARIS_SWEEP_PAIRS"] = "0"   # the TMA staging is a form of the single sweep
    try:
        with runtime.ParisGpu(desc) as gpu:
            gpu.upload(capi.F_CVOF, cvof)
            for f, a in zip((capi.F_U, capi.F_V, capi.F_W), vel):
                gpu.upload(f, a)
            gpu.linfunc(capi.F_RHO)
            gpu.setup_poisson(1e-3)
            gpu.fill_field(capi.F_P, 0.0)
            r = gpu.new_solver(0.0, maxit=6, mode=capi.MG_MIXED, rel_tol=1e-300, pcg=pcg)
            return gpu.download(capi.F_P), r
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("pcg", [0, 1])
@pytest.mark.parametrize("n,bc", [((64, 64, 64), "periodic"), ((64, 64, 64), "wall"),
                                  ((128, 64, 64), (1, 0, 1, 1, 0, 1)), ((64, 128, 64), (0, 1, 0, 0, 1, 0)),
                                  ((128, 128, 128), "periodic")])
def test_tma_sweep_matches_cp_async(gpu_lib, capi, runtime, orc, workloads, n, bc, pcg):
    desc, cvof, vel = _problem(capi, orc, workloads, n, bc, seed=5)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p_tma, r_tma = _solve(runtime, capi, desc, cvof, vel, True, pcg)
        p_cpa, r_cpa = _solve(runtime, capi, desc, cvof, vel, False, pcg)
    assert_same_solve(p_tma, r_tma, p_cpa, r_cpa, pcg, True)

