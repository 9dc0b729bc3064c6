"""The device step with DoMOMCONS on the reference's Tests/CylinderAdvection
case (16 x 16 x 2 periodic, elliptic cylinder of density 1e5 in density 1,
uniform velocity (0.01, 0.01, 0), dt = 0.1, 3800 steps, staggered
Weymouth-Yue sweeps): the mid-plane cvof against the reference's printed
output (tests/golden/cylinder_advection_cvof.txt) to its five digits.  The
initial field is the oracle's levelset2vof of the cylinder, uploaded."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_cylinder_advection_on_the_device(gpu_lib, capi, runtime, orc):
    with open(os.path.join(HERE, "golden", "cylinder_advection_cvof.txt")) as f:
        ref = np.array([float(x) for x in f if x.strip() and not x.startswith("#")]).reshape(16, 16)
    d = capi.make_desc((16, 16, 2), length=(1.0, 1.0, 0.125), bc="periodic", rho1=1.0, rho2=1e5, mu1=0.0,
                       mu2=0.0, sigma=0.0)
    d.vof_advect = capi.ADVECT_WY
    cvof, flag, _ = orc.init_shapes(d, [(0.5, 0.5, 0.5)], [0.1], excentricity=(1.0, 0.0, 0.0), ipar=-3)
    solve = {"max_error": 1e-5, "rel_tol": 0.0, "maxit": 200, "mode": capi.MG_MIXED, "pcg": 1}
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        for f in (capi.F_U, capi.F_V):
            gpu.fill_field(f, 0.01)
        for f in (capi.F_W, capi.F_P):
            gpu.fill_field(f, 0.0)
        for k in range(1, 3801):
            gpu.ns_step(k, 0.1, solve=solve, momcons={"staggered": True})
        out = gpu.download(capi.F_CVOF)
        u, v, w = (gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W))
    g = d.ng
    got = out[g, g:-g, g:-g].T
    mag = np.floor(np.log10(np.where(ref == 0.0, 1.0, np.abs(ref))))
    tol = np.where(ref == 0.0, 1e-12, 0.5 * 10.0 ** (mag - 4) * (1.0 + 1e-6))
    err = np.abs(got - ref)
    print(f"\ncylinder advection on the device: max |cvof - reference| {err.max():.3e}")
    assert (err <= tol).all(), (np.argwhere(err > tol)[:5], got[err > tol][:5], ref[err > tol][:5])
    assert np.abs(u - 0.01).max() < 1e-13 and np.abs(v - 0.01).max() < 1e-13 and np.abs(w).max() < 1e-13
