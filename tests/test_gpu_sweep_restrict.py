"""The last pre-smoothing sweep fused with the restriction against the sweep
followed by the restriction kernel.

k_rb_sweep_rs performs the sweep of k_rb_sweep2_cfg and forms the residual and
the coarse right-hand side with the operations of k_fast_restrict2 in the
same order, so a solve with either gives the same pressure to the bit.  The
environment variable PARIS_SWEEP_RS, read when a handle first builds its
multigrid levels, selects the fused form on the finest level (1), on every
fused level (2), or nowhere (0, the default).  The FP32 cycle of the
mixed solver, both outer loops, on periodic, walled and mixed boxes whose
levels do not all fit the 32 x 8 tiles in whole numbers, with the smoother
over-relaxed (1.1) or not."""
import os
import warnings

import numpy as np
import pytest

from sweep_case import problem

pytestmark = pytest.mark.gpu


def _solve(runtime, capi, desc, cvof, vel, rs, pcg, beta):
    old = os.environ.get("PARIS_SWEEP_RS")
    os.environ["PARIS_SWEEP_RS"] = str(rs)
    try:
        with runtime.ParisGpu(desc) as gpu:
            gpu.upload(capi.F_CVOF, cvof)
            for f, a in zip((capi.F_U, capi.F_V, capi.F_W), vel):
                gpu.upload(f, a)
            gpu.linfunc(capi.F_RHO)
            gpu.setup_poisson(1e-3)
            gpu.fill_field(capi.F_P, 0.0)
            r = gpu.new_solver(0.0, beta=beta, maxit=5, mode=capi.MG_MIXED, rel_tol=1e-300, pcg=pcg,
                               nu_coarse=4, coarse_from=1, coarse_to=2)
            return gpu.download(capi.F_P), r
    finally:
        if old is None:
            del os.environ["PARIS_SWEEP_RS"]
        else:
            os.environ["PARIS_SWEEP_RS"] = old


@pytest.mark.parametrize("beta", [1.0, 1.1])
@pytest.mark.parametrize("pcg", [0, 1])
@pytest.mark.parametrize("n,bc", [((64, 64, 64), "periodic"), ((64, 64, 64), "wall"),
                                  ((96, 48, 80), (1, 0, 1, 1, 0, 1)), ((64, 112, 64), (0, 1, 0, 0, 1, 0)),
                                  ((128, 128, 128), "periodic")])
def test_fused_restriction_matches_restriction_kernel(gpu_lib, capi, runtime, orc, workloads, n, bc, pcg, beta):
    desc, cvof, vel = problem(capi, orc, workloads, n, bc, seed=17)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p0, r0 = _solve(runtime, capi, desc, cvof, vel, 0, pcg, beta)
        p1, r1 = _solve(runtime, capi, desc, cvof, vel, 1, pcg, beta)
        p2, r2 = _solve(runtime, capi, desc, cvof, vel, 2, pcg, beta)
    for p, r in ((p1, r1), (p2, r2)):
        assert r.it == r0.it
        assert r.rel_res == r0.rel_res
        assert np.array_equal(p, p0)
