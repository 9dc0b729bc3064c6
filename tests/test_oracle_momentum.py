"""Properties of the oracle's momentum predictor (no GPU needed): the
discrete operators of momentumConvection, explicitMomDiff, volumeForce and
SetVelocityBC must vanish or reproduce exactly what the continuous ones do
on the fields where the schemes are exact."""
import numpy as np
import pytest


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
def test_uniform_flow_has_no_convection(capi, orc, scheme):
    d = capi.make_desc((12, 10, 8))
    u, v, w = (orc.zeros(d) + c for c in (0.7, -0.3, 0.2))
    du, dv, dw = (orc.zeros(d) + 5.0 for _ in range(3))
    orc.momentum_convection(d, scheme, u, v, w, du, dv, dw)
    for a in (du, dv, dw):
        assert np.abs(orc.interior(d, a)).max() < 1e-12


def test_linear_shear_has_no_viscous_force(capi, orc):
    """u = a*y + b*z with constant mu: every second difference vanishes."""
    n = 12
    d = capi.make_desc((n, n, n), bc="wall")
    c = orc.grid_coords(d)
    Y = c["y"][None, :, None] + 0 * c["x"][None, None, :]
    Z = c["z"][:, None, None] + 0 * Y
    u = 0.4 * Y + 0.2 * Z + 0 * Z
    v, w = orc.zeros(d), orc.zeros(d)
    rho, mu = orc.zeros(d) + 2.0, orc.zeros(d) + 1e-2
    du, dv, dw = (orc.zeros(d) for _ in range(3))
    orc.explicit_mom_diff(d, u, v, w, rho, mu, du, dv, dw)
    g = d.ng
    for a in (du, dv, dw):
        assert np.abs(a[g + 1:-g - 1, g + 1:-g - 1, g + 1:-g - 1]).max() < 1e-13


def test_gravity_on_uniform_density(capi, orc):
    d = capi.make_desc((8, 8, 8), bc="wall", rho1=1.0, rho2=3.0)
    rho = orc.zeros(d) + 3.0
    du, dv, dw = (orc.zeros(d) for _ in range(3))
    orc.volume_force(d, rho, du, dv, dw, buoyancy=0, gz=-9.81)
    g = d.ng
    assert np.all(orc.interior(d, du)[:, :, :-1] == 0.0)
    assert np.all(dw[g:g + 7, g:-g, g:-g] == -9.81)
    # buoyancy relative to the heavy phase removes it
    du, dv, dw = (orc.zeros(d) for _ in range(3))
    orc.volume_force(d, rho, du, dv, dw, buoyancy=2, gz=-9.81)
    assert np.all(dw == 0.0)


def test_walls_stop_the_normal_flow(capi, orc):
    n = 10
    d = capi.make_desc((n, n, n), bc="wall")
    rng = np.random.default_rng(0)
    u, v, w = (rng.standard_normal(orc.shape(d)) for _ in range(3))
    orc.set_velocity_bc(d, u, v, w)
    g = d.ng
    assert np.all(u[g:-g, g:-g, g - 1] == 0.0) and np.all(u[g:-g, g:-g, g + n - 1] == 0.0)
    assert np.all(v[g:-g, g - 1, g:-g] == 0.0) and np.all(w[g - 1, g:-g, g:-g] == 0.0)
    # resting walls: the tangential velocity is odd across the wall
    assert np.array_equal(v[g:-g, g:-g, g - 1], -v[g:-g, g:-g, g])
