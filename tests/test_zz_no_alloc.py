"""The allocation-free residual entry point, for callers that cannot
allocate device memory (their device memory belongs to their own pool or to
another runtime, or they run under a fixed budget).  It must give the same
L1/L2/Linf as the handle-based calcResiduals, on two calls in a row (the
second call reuses the shared scratch array left by the first).

This file is collected last so that a run stopping at its first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_calc_residuals_noalloc_matches(gpu_lib, capi, runtime, orc, workloads):
    import torch

    n = 24
    desc = capi.make_desc((n, n, n), rho1=1.0, rho2=1000.0)
    cen, rad = workloads.drop_layout(4, rmin=0.1, rmax=0.2, seed=3, h=1.0 / n)
    cvof, _, _ = orc.init_spheres(desc, cen, rad, refinement=4)
    rho = orc.linfunc(desc, cvof, 1.0, 1000.0, capi.MEAN_ARITH)
    rng = np.random.default_rng(11)
    vel = []
    for _ in range(3):
        f = orc.zeros(desc)
        orc.interior(desc, f)[...] = rng.standard_normal((n, n, n))
        orc.fill_ghosts(desc, f)
        vel.append(f)
    _, A = orc.setup_poisson(desc, *vel, rho, 1e-3)
    p1 = orc.zeros(desc)
    orc.interior(desc, p1)[...] = rng.standard_normal((n, n, n))
    orc.fill_ghosts(desc, p1)
    p2 = p1 * 0.5 + 1.0

    lib = gpu_lib
    stream = torch.cuda.current_stream()
    A_dev = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    for call, p in enumerate((p1, p2)):
        with runtime.ParisGpu(desc) as gpu:
            gpu.upload(capi.F_A, A)
            gpu.upload(capi.F_P, p)
            want = gpu.calc_residuals()
        p_dev = torch.from_numpy(np.ascontiguousarray(p)).cuda()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        out = np.zeros(3)
        st = lib.paris_calc_residuals_noalloc(n, n, n, desc.ng, ctypes.c_void_p(A_dev.data_ptr()),
                                              ctypes.c_void_p(p_dev.data_ptr()),
                                              out.ctypes.data_as(ctypes.c_void_p),
                                              ctypes.c_void_p(stream.cuda_stream))
        assert st == capi.OK
        if call == 1:   # the module is loaded by now: no device memory is taken
            assert torch.cuda.mem_get_info()[0] == free0
        np.testing.assert_allclose(out[:2], want[:2], rtol=1e-12)
        assert out[2] == want[2]
        # calcResiduals of the oracle (modules.f90:3313-3387): L1, L2, Linf
        ref = [orc.calc_residual(desc, A, p, k) for k in (1, 2, 3)]
        np.testing.assert_allclose(out, ref, rtol=1e-12)


def test_calc_residuals_noalloc_rejects_oversize(gpu_lib, capi):
    out = np.zeros(3)
    dummy = ctypes.c_void_p(16)
    st = gpu_lib.paris_calc_residuals_noalloc(512, 256, 256, 2, dummy, dummy, out.ctypes.data_as(ctypes.c_void_p),
                                              None)
    assert st == capi.BAD_ARGS
