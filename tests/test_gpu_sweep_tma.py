"""The TMA-staged fused sweep against the cp.async-staged one.

The two kernels share the tiles, the wavefront and the arithmetic of the
fused red-black sweep and differ only in how the planes reach shared memory,
so a solve with either must give the same pressure to the bit.  The
environment variable PARIS_SWEEP_TMA, read when a handle first builds its
FP32 multigrid levels, selects the TMA staging (1) or the cp.async one (0,
the default).  Grids: periodic and
walled boxes, and mixed boundaries, whose fused levels (at least 64^3 cells)
have the first and last tiles of every row and column wrapped or zero."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(capi, orc, workloads, n, bc, seed):
    desc = capi.make_desc(n, bc=bc, rho1=1.0, rho2=1000.0)
    cen, rad = workloads.drop_layout(6, rmin=0.1, rmax=0.2, seed=seed, h=1.0 / max(n))
    cvof, _, _ = orc.init_spheres(desc, cen, rad, refinement=2)
    rng = np.random.default_rng(seed)
    vel = []
    for d in range(3):
        f = orc.zeros(desc)
        orc.interior(desc, f)[...] = rng.standard_normal((n[2], n[1], n[0]))
        orc.fill_ghosts(desc, f)
        vel.append(f)
    g = desc.ng
    per = [bc == "periodic" or (not isinstance(bc, str) and bc[a] == 1) for a in range(3)]
    if not per[0]:
        vel[0][:, :, g - 1] = 0.0
        vel[0][:, :, g + n[0] - 1] = 0.0
    if not per[1]:
        vel[1][:, g - 1, :] = 0.0
        vel[1][:, g + n[1] - 1, :] = 0.0
    if not per[2]:
        vel[2][g - 1, :, :] = 0.0
        vel[2][g + n[2] - 1, :, :] = 0.0
    return desc, cvof, vel


def _solve(runtime, capi, desc, cvof, vel, tma, pcg):
    old = os.environ.get("PARIS_SWEEP_TMA")
    os.environ["PARIS_SWEEP_TMA"] = "1" if tma else "0"
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
        if old is None:
            del os.environ["PARIS_SWEEP_TMA"]
        else:
            os.environ["PARIS_SWEEP_TMA"] = old


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
    assert r_tma.it == r_cpa.it
    assert r_tma.rel_res == r_cpa.rel_res
    assert np.array_equal(p_tma, p_cpa)

