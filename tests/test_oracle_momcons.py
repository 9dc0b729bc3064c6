"""Oracle of the momentum-conserving VOF sweeps (DoMOMCONS) on the CPU: the
flux centroid against sampled and closed-form centroids, and properties of
the sweeps that hold whatever the geometry: a uniform velocity stays
uniform (the momentum flux is the velocity times the mass flux), and the
Weymouth-Yue sweeps conserve the total momentum of a periodic box when the
velocity is uniform."""
import numpy as np
import pytest


def test_flux_centroid_closed_forms(orc):
    # a corner tetrahedron: centroid at a quarter of the intercepts
    nr, al = np.array([0.3, 0.3, 0.4]), 0.2
    assert np.allclose(orc.flux_centroid(nr, al, [0, 0, 0], [1, 1, 1]), [al / 4 / 0.3, al / 4 / 0.3, al / 4 / 0.4],
                       rtol=1e-14)
    # a slab x < 0.5
    assert np.allclose(orc.flux_centroid([1, 0, 0], 0.5, [0, 0, 0], [1, 1, 1]), [0.25, 0.5, 0.5], rtol=1e-14)
    # a shifted, stretched box with a negative coefficient: the slab x > 0.3 of [0.2, 0.5]
    assert np.allclose(orc.flux_centroid([-1, 0, 0], -0.3, [0.2, 0, 0], [0.3, 1, 1]), [0.4, 0.5, 0.5], rtol=1e-14)


@pytest.mark.parametrize("nr,al", [([0.3, 0.3, 0.4], 0.45), ([0.1, 0.2, 0.7], 0.35), ([0.2, 0.5, 0.3], 0.7),
                                   ([-0.3, 0.5, 0.2], 0.1), ([0.45, 0.05, 0.5], 0.6)])
def test_flux_centroid_against_samples(orc, nr, al):
    """The five cases of the plane position (and the complement above one
    half) against the mean of 2 million seeded points of the cut box."""
    rng = np.random.default_rng(7)
    x0, dx = np.array([0.1, 0.0, 0.2]), np.array([0.6, 1.0, 0.5])
    p = x0 + dx * rng.random((2_000_000, 3))
    inside = p @ np.asarray(nr) < al
    want = p[inside].mean(axis=0)
    got = orc.flux_centroid(nr, al, x0, dx)
    assert np.abs(got - want).max() < 2e-3 * dx.max(), (got, want)


def _state(capi, orc, n, advect, bc="periodic", seed=3, uniform=None, rho=(1.0, 10.0)):
    d = capi.make_desc((n, n, n), bc=bc, rho1=rho[0], rho2=rho[1])
    d.vof_advect = advect
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0.25, 0.75, (3, 3))
    cvof, flag, _ = orc.init_spheres(d, cen, rng.uniform(0.1, 0.2, 3), refinement=4)
    if uniform is not None:
        u, v, w = (np.full(orc.shape(d), uniform[a]) for a in range(3))
    else:
        u, v, w = (0.3 * rng.standard_normal(orc.shape(d)) for _ in range(3))
        for a in (u, v, w):
            orc.fill_ghosts(d, a)
    return d, cvof, flag, u, v, w


@pytest.mark.parametrize("staggered", [True, False])
@pytest.mark.parametrize("advect", ["CIAM", "WY"])
@pytest.mark.parametrize("lin", [False, True])
def test_uniform_velocity_stays_uniform(capi, orc, staggered, advect, lin):
    if lin and not staggered:
        pytest.skip("LinInterp belongs to the staggered sweeps")
    n, U = 16, (0.7, -0.4, 0.25)
    d, cvof, flag, u, v, w = _state(capi, orc, n, capi.ADVECT_CIAM if advect == "CIAM" else capi.ADVECT_WY,
                                    uniform=U)
    dt = 0.3 / n / 0.7
    du, dv, dw = (np.full(orc.shape(d), 5.0) for _ in range(3))
    mom = orc.zeros(d)
    orc.vof_mom_sweeps(d, 1, dt, cvof, flag, u, v, w, du, dv, dw, mom, staggered=staggered, lin_interp=lin)
    g = d.ng
    inner = (slice(g, -g),) * 3
    for a, comp in zip((du, dv, dw), U):
        touched = a[inner] != 5.0
        assert touched.any()
        # (mom/rho - U)/dt where the advected fraction is mixed: round-off of U/dt only
        assert np.abs(a[inner][touched]).max() * dt < 1e-9 * max(abs(x) for x in U), np.abs(a[inner][touched]).max()


def test_wy_conserves_momentum_of_a_periodic_box(capi, orc):
    """Weymouth-Yue fluxes with a uniform velocity: every flux leaves one
    cell and enters its neighbour, and the central term vanishes."""
    n = 16
    d, cvof, flag, u, v, w = _state(capi, orc, n, capi.ADVECT_WY, uniform=(0.5, 0.3, -0.2))
    dt = 0.4 / n / 0.5
    du, dv, dw = (orc.zeros(d) for _ in range(3))
    mom = orc.zeros(d)
    g = d.ng
    inner = (slice(g, -g),) * 3
    orc.vof_mom_sweeps(d, 2, dt, cvof, flag, u, v, w, du, dv, dw, mom, staggered=True)
    # the staggered fraction of w is the average of the upper half of k and
    # the lower half of k+1, so its total is the total of cvof; the momentum
    # total is then w (rho1 N + (rho2 - rho1) sum cvof)
    total = float(mom[inner].sum())
    want = -0.2 * (d.rho1 * n ** 3 + (d.rho2 - d.rho1) * float(cvof[inner].sum()))
    assert abs(total - want) <= 1e-11 * abs(want), (total, want)


def test_rejects_unsupported_boundaries(capi, orc):
    d, cvof, flag, u, v, w = _state(capi, orc, 8, capi.ADVECT_CIAM)
    d.bdry_cond[0] = capi.BC_SHEAR
    du, dv, dw = (orc.zeros(d) for _ in range(3))
    with pytest.raises(AssertionError):
        orc.vof_mom_sweeps(d, 0, 1e-3, cvof, flag, u, v, w, du, dv, dw, orc.zeros(d))


def test_init_shapes_cylinders_and_spheres(capi, orc):
    """levelset2vof(shapes2ls, ipar): a cylinder along each axis with an
    excentricity has the area pi a b of its ellipse per unit length (to the
    refinement's accuracy), and spheres without excentricity are the
    init_spheres fields bit for bit."""
    n = 32
    d = capi.make_desc((n, n, n))
    g = d.ng
    for axis in range(3):
        exc = [0.0, 0.0, 0.0]
        exc[(axis + 1) % 3] = 1.0   # semi-axis sqrt(2) R along the next axis
        cvof, flag, _ = orc.init_shapes(d, [(0.5, 0.5, 0.5)], [0.2], excentricity=exc, ipar=-(axis + 1))
        vol = cvof[g:-g, g:-g, g:-g].sum() / n ** 3
        assert abs(vol - np.pi * 0.2 * 0.2 * np.sqrt(2.0)) < 2e-3, (axis, vol)
        c = cvof[g:-g, g:-g, g:-g]
        assert np.array_equal(c, np.moveaxis(np.moveaxis(c, 2 - axis, 0)[[0] * n], 0, 2 - axis)), axis
    cen = [(0.3, 0.4, 0.5), (0.7, 0.6, 0.45)]
    a = orc.init_shapes(d, cen, [0.12, 0.1])
    b = orc.init_spheres(d, cen, [0.12, 0.1])
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
