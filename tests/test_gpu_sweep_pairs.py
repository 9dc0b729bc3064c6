"""Two smoothing sweeps in one pass against the same sweeps one at a time.

k_rb_sweep4_cfg runs the two red-black sweeps of a V(2,2) smoothing pass in
one pass over memory; every cell update reads the same neighbour values as in
two calls of the single fused sweep, with the same arithmetic, so a
defect-correction solve with either form gives the same pressure to the bit
(and a CG solve the same to rounding: assert_same_solve).  The environment variable
PARIS_SWEEP_PAIRS, read when a handle first builds its multigrid levels,
selects the pair form (1) or single sweeps (0).  Both the FP32 inner cycle of
the mixed solver and the FP64 solver, with and without the CG outer loop, on
periodic, walled and mixed boxes whose fused levels (at least 32^3 cells) do
not all fit the tiles in whole numbers."""
import os
import warnings

import numpy as np
import pytest

from sweep_case import assert_same_solve, problem

pytestmark = pytest.mark.gpu


def _solve(runtime, capi, desc, cvof, vel, pairs, mode, pcg, nu=2, beta=1.0):
    old = os.environ.get("PARIS_SWEEP_PAIRS")
    os.environ["PARIS_SWEEP_PAIRS"] = "1" if pairs else "0"
    try:
        with runtime.ParisGpu(desc) as gpu:
            gpu.upload(capi.F_CVOF, cvof)
            for f, a in zip((capi.F_U, capi.F_V, capi.F_W), vel):
                gpu.upload(f, a)
            gpu.linfunc(capi.F_RHO)
            gpu.setup_poisson(1e-3)
            gpu.fill_field(capi.F_P, 0.0)
            r = gpu.new_solver(0.0, beta=beta, maxit=5, mode=mode, rel_tol=1e-300, pcg=pcg, nu1=nu, nu2=nu)
            return gpu.download(capi.F_P), r
    finally:
        if old is None:
            del os.environ["PARIS_SWEEP_PAIRS"]
        else:
            os.environ["PARIS_SWEEP_PAIRS"] = old


@pytest.mark.parametrize("pcg", [0, 1])
@pytest.mark.parametrize("mode", ["mixed", "fp64"])
@pytest.mark.parametrize("n,bc", [((64, 64, 64), "periodic"), ((64, 64, 64), "wall"),
                                  ((96, 48, 80), (1, 0, 1, 1, 0, 1)), ((64, 112, 64), (0, 1, 0, 0, 1, 0)),
                                  ((128, 128, 128), "periodic")])
def test_pair_sweep_matches_single_sweeps(gpu_lib, capi, runtime, orc, workloads, n, bc, mode, pcg):
    desc, cvof, vel = problem(capi, orc, workloads, n, bc, seed=7)
    m = capi.MG_MIXED if mode == "mixed" else capi.MG_FP64
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p_pair, r_pair = _solve(runtime, capi, desc, cvof, vel, True, m, pcg)
        p_one, r_one = _solve(runtime, capi, desc, cvof, vel, False, m, pcg)
    assert_same_solve(p_pair, r_pair, p_one, r_one, pcg, mode == "mixed")


@pytest.mark.parametrize("nu", [1, 3, 4])
def test_pair_sweep_odd_and_repeated_passes(gpu_lib, capi, runtime, orc, workloads, nu):
    """V(1,1): single sweeps only; V(3,3): a pair and a single sweep (the pair
    first, with the coarse correction after the coarse level); V(4,4): two
    pairs, the second without it.  CG outer loop."""
    desc, cvof, vel = problem(capi, orc, workloads, (64, 64, 64), (1, 0, 1, 1, 0, 1), seed=11)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p_pair, r_pair = _solve(runtime, capi, desc, cvof, vel, True, capi.MG_MIXED, 1, nu)
        p_one, r_one = _solve(runtime, capi, desc, cvof, vel, False, capi.MG_MIXED, 1, nu)
    assert_same_solve(p_pair, r_pair, p_one, r_one, 1, True)


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_pair_sweep_over_relaxed(gpu_lib, capi, runtime, orc, workloads, mode):
    """With the smoother over-relaxed (the solver's beta, here 1.15) the two
    forms still read the same values: the same pressure to the bit by defect
    correction, to rounding by CG."""
    desc, cvof, vel = problem(capi, orc, workloads, (96, 48, 80), (1, 0, 1, 1, 0, 1), seed=13)
    m = capi.MG_MIXED if mode == "mixed" else capi.MG_FP64
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p_pair, r_pair = _solve(runtime, capi, desc, cvof, vel, True, m, 1, beta=1.15)
        p_one, r_one = _solve(runtime, capi, desc, cvof, vel, False, m, 1, beta=1.15)
    assert_same_solve(p_pair, r_pair, p_one, r_one, 1, mode == "mixed")
    p_pair, r_pair = _solve(runtime, capi, desc, cvof, vel, True, m, 0, beta=1.15)
    p_one, r_one = _solve(runtime, capi, desc, cvof, vel, False, m, 0, beta=1.15)
    assert_same_solve(p_pair, r_pair, p_one, r_one, 0, mode == "mixed")
