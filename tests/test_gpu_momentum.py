"""The explicit momentum predictor on the GPU against the FP64 oracle, bit for
bit: momentumConvection (QUICK, ENO, Superbee, WENO), explicitMomDiff,
volumeForce, u = u + dt*du and SetVelocityBC (walls with moving-wall
velocities, periodic images).  All kernels keep the Fortran operation order
(no FMA contraction), so the comparison is exact, ghost entries included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fields(capi, orc, n, bc, seed, grid="general"):
    # "pow2": 16^3 on the unit cube, where the QUICK kernel multiplies by the
    # exact reciprocals of its powers of two; "general": 16x20x14 (cells of
    # 1/20 and 1/14 along y and z), where it divides
    shape = (n, n, n) if grid == "pow2" else (n, n + 4, n - 2)
    d = capi.make_desc(shape, bc=bc, rho1=1.2, rho2=1000.0, mu1=1.7e-5, mu2=1e-3)
    rng = np.random.default_rng(seed)
    u, v, w = (rng.standard_normal(orc.shape(d)) for _ in range(3))
    orc.set_velocity_bc(d, u, v, w)          # consistent ghosts (walls: reflected, periodic: images)
    rho = orc.zeros(d) + rng.uniform(1.0, 1000.0, orc.shape(d))
    mu = orc.zeros(d) + rng.uniform(1e-5, 1e-3, orc.shape(d))
    return d, u, v, w, rho, mu


def upload(gpu, capi, **kw):
    for name, a in kw.items():
        gpu.upload(getattr(capi, "F_" + name.upper()), a)


@pytest.mark.parametrize("grid", ["general", "pow2"])
@pytest.mark.parametrize("bc", ["periodic", "wall"])
@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
def test_convection_bitwise(gpu_lib, capi, runtime, orc, bc, scheme, grid):
    d, u, v, w, rho, mu = fields(capi, orc, 16, bc, 1, grid)
    sentinel = [orc.zeros(d) + 7.0 + q for q in range(3)]   # entries the scheme leaves alone stay
    ref = [a.copy() for a in sentinel]
    assert orc.momentum_convection(d, scheme, u, v, w, *ref) == 0
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, u=u, v=v, w=w, du=sentinel[0], dv=sentinel[1], dw=sentinel[2])
        gpu.momentum_convection(scheme)
        out = [gpu.download(f) for f in (capi.F_DU, capi.F_DV, capi.F_DW)]
    for a, b, s in zip(out, ref, sentinel):
        assert np.array_equal(a, b)
        assert (b != s).any()


@pytest.mark.parametrize("grid", ["general", "pow2"])
@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_diffusion_force_advance_bitwise(gpu_lib, capi, runtime, orc, bc, grid):
    d, u, v, w, rho, mu = fields(capi, orc, 16, bc, 2, grid)
    rng = np.random.default_rng(3)
    du, dv, dw = (rng.standard_normal(orc.shape(d)) for _ in range(3))
    ref = [a.copy() for a in (du, dv, dw)]
    orc.explicit_mom_diff(d, u, v, w, rho, mu, *ref)
    orc.volume_force(d, rho, *ref, dpdx=0.3, dpdy=-0.1, dpdz=0.05, buoyancy=1, gx=0.0, gy=0.0, gz=-9.81)
    uu = [a.copy() for a in (u, v, w)]
    orc.advance_velocity(d, 1e-3, *uu, *ref)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, u=u, v=v, w=w, rho=rho, mu=mu, du=du, dv=dv, dw=dw)
        gpu.explicit_mom_diff()
        gpu.volume_force(dpdx=0.3, dpdy=-0.1, dpdz=0.05, buoyancy=1, gz=-9.81)
        mid = [gpu.download(f) for f in (capi.F_DU, capi.F_DV, capi.F_DW)]
        gpu.advance_velocity(1e-3)
        out = [gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W)]
    for a, b in zip(mid, ref):
        assert np.array_equal(a, b)
    for a, b in zip(out, uu):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("bc", ["periodic", "wall", "mixed"])
def test_velocity_bc_bitwise(gpu_lib, capi, runtime, orc, bc):
    n = 12
    if bc == "mixed":   # periodic in x, walls in y and z
        P, W = capi.BC_PERIODIC, capi.BC_WALL
        d = capi.make_desc((n, n, n), bc=[P, W, W, P, W, W])
    else:
        d = capi.make_desc((n, n, n), bc=bc)
    rng = np.random.default_rng(4)
    u, v, w = (rng.standard_normal(orc.shape(d)) for _ in range(3))
    wall = rng.standard_normal((6, 3))
    ref = [a.copy() for a in (u, v, w)]
    orc.set_velocity_bc(d, *ref, wall_vel=wall)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, u=u, v=v, w=w)
        gpu.set_velocity_bc(wall)
        out = [gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W)]
    for a, b in zip(out, ref):
        assert np.array_equal(a, b)
    if bc != "periodic":
        g = d.ng
        # no flow through the walls, and the tangential velocity averages to
        # the wall's across the wall (x- and z- faces)
        assert np.all(out[1][g:-g, g - 1, :] == 0.0)
        avg = 0.5 * (out[0][g - 1, g:-g, g:-g] + out[0][g, g:-g, g:-g])
        assert np.allclose(avg, wall[4, 0], atol=1e-14)
