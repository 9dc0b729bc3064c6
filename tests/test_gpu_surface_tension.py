"""Parity of the height functions, curvature and CSF force on the GPU
against the FP64 oracle.

Heights are sums of volume fractions in the reference's order: they must be
equal bit for bit.  Curvatures go through AL3D (pow/acos/cos) and 6x6
Gauss-Jordan fits, where the device and glibc transcendental functions may
differ by an ulp: the same cells must get a curvature, by the same method,
and the values agree to 1e-9 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KAPPA_RTOL = 1e-9


def layouts(orc, capi, case):
    if case == "sphere":
        n = 32
        d = capi.make_desc((n, n, n), do_rotation=1)
        cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [0.32], refinement=8)
    elif case == "seam":
        # a drop straddling the periodic boundary in x (and its image)
        n = 32
        d = capi.make_desc((n, n, n))
        cvof, flag, _ = orc.init_spheres(d, [(0.03, 0.45, 0.52), (1.03, 0.45, 0.52), (0.6, 0.6, 0.35)],
                                         [0.2, 0.2, 0.17], refinement=4)
    elif case == "walls":
        n = 24
        d = capi.make_desc((n, n, n), bc="wall")
        cvof, flag, _ = orc.init_spheres(d, [(0.45, 0.5, 0.3), (0.6, 0.55, 0.72)], [0.2, 0.16], refinement=4)
    elif case == "tiny":
        # drops of about 1.5-2 cells radius: centroid fits and averages
        n = 24
        d = capi.make_desc((n, n, n))
        cen = [(0.3, 0.3, 0.3), (0.7, 0.33, 0.6), (0.45, 0.72, 0.45), (0.2, 0.75, 0.8)]
        cvof, flag, _ = orc.init_spheres(d, cen, [0.07, 0.063, 0.077, 0.07], refinement=4)
    else:
        n = 40
        d = capi.make_desc((n, n, n))
        cen = [(0.3, 0.3, 0.3), (0.7, 0.35, 0.6), (0.45, 0.72, 0.45), (0.2, 0.75, 0.8)]
        cvof, flag, _ = orc.init_spheres(d, cen, [0.12, 0.1, 0.15, 0.08], refinement=4)
    return d, cvof, flag


@pytest.mark.parametrize("case", ["sphere", "seam", "walls", "drops", "tiny"])
def test_heights_and_curvature(gpu_lib, capi, runtime, orc, case):
    d, cvof, flag = layouts(orc, capi, case)
    H_ref = orc.get_all_heights(d, cvof, flag)
    kap_ref, kf_ref, mc = orc.get_all_curvatures(d, cvof, flag, H_ref)
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        gpu.get_all_heights()
        H = gpu.download(capi.F_HEIGHT)
        kap = gpu.get_all_curvatures()
    assert np.array_equal(H, H_ref)
    valid_ref = kap_ref < 1e6
    assert np.array_equal(kap < 1e6, valid_ref)
    scale = np.abs(kap_ref[valid_ref]).max()
    assert np.abs(kap[valid_ref] - kap_ref[valid_ref]).max() <= KAPPA_RTOL * scale
    assert mc.sum() > 0


@pytest.mark.parametrize("case", ["sphere", "walls", "tiny"])
def test_surface_force(gpu_lib, capi, runtime, orc, case):
    d, cvof, flag = layouts(orc, capi, case)
    d.sigma = 0.7
    d.rho1, d.rho2 = 1.0, 1000.0
    rho = orc.linfunc(d, cvof, d.rho1, d.rho2, capi.MEAN_ARITH)
    H_ref = orc.get_all_heights(d, cvof, flag)
    kap_ref, _, _ = orc.get_all_curvatures(d, cvof, flag, H_ref)
    rng = np.random.default_rng(2)
    du0 = [rng.standard_normal(orc.shape(d)) for _ in range(3)]
    ref = [a.copy() for a in du0]
    orc.surface_force(d, cvof, kap_ref, rho, *ref)
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        gpu.upload(capi.F_RHO, rho)
        for f, a in zip((capi.F_DU, capi.F_DV, capi.F_DW), du0):
            gpu.upload(f, a)
        gpu.get_all_heights()
        gpu.surface_force()
        out = [gpu.download(f) for f in (capi.F_DU, capi.F_DV, capi.F_DW)]
    for a, b, a0 in zip(out, ref, du0):
        changed = b != a0
        assert changed.any()
        assert np.array_equal(a != a0, changed)
        scale = np.abs(b - a0).max()
        assert np.abs(a - b).max() <= KAPPA_RTOL * scale
