"""Properties of the oracle's time-step control and flow statistics (no GPU
needed): TimeStepSize and get_cfl_and_check (paris.f90:968-1074) and the
calcStats columns (paris.f90:1116-1267) on fields where each column is known
in closed form."""
import math

import numpy as np
import pytest


def fields(capi, orc, d):
    z = {k: orc.zeros(d) for k in ("u", "v", "w", "rho", "p", "cvof", "mu")}
    z["flag"] = orc.zeros(d, np.int32)
    return z


def stats(orc, d, f, opts=None):
    return orc.calc_stats(d, f["u"], f["v"], f["w"], f["rho"], f["p"], f["cvof"], f["mu"], f["flag"], opts)


def test_time_step_size_and_cfl(capi, orc):
    n = 16
    d = capi.make_desc((n, n, n), bc="wall")
    f = fields(capi, orc, d)
    h = 1.0 / n
    # at rest the physical floor vmax_phys = 1e-3 sets dt, clamped by MaxDt
    dt, vmax = orc.time_step_size(d, f["u"], f["v"], f["w"], 0.5, 1e9)
    assert vmax == 0.0 and dt == 0.5 * (h / 1e-3)
    dt, _ = orc.time_step_size(d, f["u"], f["v"], f["w"], 0.5, 5e-2)
    assert dt == 5e-2
    # one cell moving: vmax is sqrt(u^2+v^2+w^2) at the same (i,j,k); ghosts ignored
    g = d.ng
    f["u"][g + 3, g + 4, g + 5], f["v"][g + 3, g + 4, g + 5], f["w"][g + 3, g + 4, g + 5] = 3.0, 4.0, 12.0
    f["u"][0, 0, 0] = 1e6
    dt, vmax = orc.time_step_size(d, f["u"], f["v"], f["w"], 0.25, 1.0)
    assert vmax == 13.0 and dt == 0.25 * (h / 13.0)
    st, cfl = orc.get_cfl_and_check(d, f["u"], f["v"], f["w"], 1e-3)
    assert st == 0 and cfl == 13.0 * 1e-3 / h
    st, cfl = orc.get_cfl_and_check(d, f["u"], f["v"], f["w"], 1e-2)
    assert st == capi.CFL_TOO_LARGE and cfl > 0.5


def test_uniform_flow_and_rotation(capi, orc):
    """u = U0 + solid-body rotation about z: every column that the central
    differences make exact."""
    n, U0, om = 12, 0.7, 1.3
    d = capi.make_desc((n, n, n), bc="periodic", rho1=2.0, rho2=2.0)
    f = fields(capi, orc, d)
    c = orc.grid_coords(d)
    f["u"][:] = U0
    f["rho"][:] = 2.0
    # solid-body rotation in the x-y plane, linear through the ghosts
    Y = c["y"][None, :, None] + 0 * c["x"][None, None, :]
    X = c["x"][None, None, :] + 0 * c["y"][None, :, None]
    f["u"] = f["u"] - om * (Y + 0 * f["u"])
    f["v"] = f["v"] + om * (X + 0 * f["v"])
    s, _ = stats(orc, d, f)
    # vorticity 2*om everywhere: enstrophy 0.5*(2 om)^2 per unit volume, all in phase 0
    assert s[22] == pytest.approx(0.5 * (2 * om) ** 2, rel=1e-12)
    assert s[21] == 0.0
    assert s[5] == pytest.approx(2.0, rel=1e-14)      # <rho>, normalised by the box volume
    assert s[9] == 0.0 and s[24] == 0.0               # no liquid, no mixed cells


def test_sphere_volume_area_and_flags(capi, orc):
    n, R = 32, 0.25
    d = capi.make_desc((n, n, n), bc="wall")
    f = fields(capi, orc, d)
    f["cvof"], f["flag"], _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [R], refinement=8)
    opts = capi.make_stats_opts(test_flags=capi.STATS_RISING_BUBBLE)
    f["u"][:] = 0.3
    s, _ = stats(orc, d, f, opts)
    vol = 4.0 / 3.0 * math.pi * R ** 3
    assert s[9] == pytest.approx(vol, rel=2e-3)       # rising bubble: the phase volume itself
    assert s[10] == pytest.approx(0.5, abs=1e-12)     # x centre of mass
    assert s[23] == pytest.approx(0.3, rel=1e-12)     # rise velocity of a uniform flow
    assert s[24] == np.count_nonzero(orc.interior(d, f["flag"]) == 2)
    area = 4.0 * math.pi * (R * n) ** 2               # AREA3D is in cell units
    assert s[18] == pytest.approx(area, rel=3e-2)
    s0, _ = stats(orc, d, f)                          # without the flag: volume fraction of the box
    assert s0[9] == pytest.approx(vol, rel=2e-3)


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_force_columns(capi, orc, bc):
    """fx, fy, fz of volumeForce on a uniform density: (rho - rro) g on the
    updated faces (all faces periodic, all but the last wall face)."""
    n = 10
    d = capi.make_desc((n, n, n), bc=bc, rho1=1.0, rho2=3.0)
    f = fields(capi, orc, d)
    f["rho"][:] = 3.0
    g = (0.5, -2.0, -9.81)
    o = capi.make_stats_opts(dpdx=(0.1, 0.0, 0.0), gravity=g, buoyancy=1)
    s, _ = stats(orc, d, f, o)
    frac = 1.0 if bc == "periodic" else (n - 1) / n
    assert s[2] == pytest.approx(frac * (-0.1 + 2.0 * g[0]), rel=1e-13)
    assert s[3] == pytest.approx(frac * 2.0 * g[1], rel=1e-13)
    assert s[4] == pytest.approx(frac * 2.0 * g[2], rel=1e-13)
    o.force_valid = 0
    s, _ = stats(orc, d, f, o)
    assert s[2] == s[3] == s[4] == 0.0
