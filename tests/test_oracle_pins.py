"""The CPU oracle checked against the reference's own regression tests and
the identities of its PLIC geometry (no GPU needed).

Pins:
  Tests/PoissonMG/run.sh:13   residual < 1e-8 and L1 error < 0.1 after 20 V-cycles
  Tests/VOF (volumeref.txt, centerofmassref.txt)   L2 tolerance 1e-4 (pariscompare)
  Tests/Curvature/run.sh:9-13  relative L2 of kappa*Nx vs -2/R < 4e-2
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_poissonmg_known_answer(capi, orc):
    d = capi.make_desc((32, 16, 16), length=(2.0, 1.0, 1.0), rho1=1.0, rho2=1e5)
    rho = orc.zeros(d) + 1.0
    A = orc.setup_testmg(d, rho)
    p = orc.zeros(d)
    st, it, tres2, hist = orc.new_solver_mg(d, A, p, 1e-300, beta=1.0, maxit=20, norm=2)
    assert it == 21 and st == capi.NOT_CONVERGED     # MAXERROR=1d-300: all 20 cycles run
    assert tres2 < 1e-8
    assert orc.mgtest_err(d, p) < 0.1
    # the residual falls monotonically, as the reference's convergence history
    assert np.all(np.diff(hist) < 0)


def _pariscompare_l2(a, b):
    """compare.c:70-96 with relative = 0: sqrt(mean (a-b)^2)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.mean((a - b) ** 2)))


def test_vof_ciam_golden(capi, orc):
    """Tests/VOF: 16^3 periodic, drop R=0.25 at the centre, u=1, dt=0.01,
    CIAM, 11 steps; stats columns 11 (volume) and 12 (x-moment)."""
    n = 16
    d = capi.make_desc((n, n, n), advect=capi.ADVECT_CIAM)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [0.25], refinement=8)
    u = orc.zeros(d) + 1.0
    v = orc.zeros(d)
    w = orc.zeros(d)
    x = orc.grid_coords(d)["x"]
    g = d.ng
    h3 = (1.0 / n) ** 3

    def stats():
        c = orc.interior(d, cvof)
        vol = c.sum() * h3
        mom = (c * x[g:g + n][None, None, :]).sum() * h3
        return vol, mom

    vols, moms = [], []
    vv, mm = stats()
    vols.append(vv)
    moms.append(mm)
    for it in range(1, 12):
        orc.vofsweeps(d, it, 0.01, cvof, flag, u, v, w)
        vv, mm = stats()
        vols.append(vv)
        moms.append(mm)
    vref = np.loadtxt(os.path.join(HERE, "golden", "vof_volumeref.txt"))[:, 1]
    mref = np.loadtxt(os.path.join(HERE, "golden", "vof_centerofmassref.txt"))[:, 1]
    # Tests/VOF/run.sh compares the last 10 volume rows and all moment rows
    got = np.concatenate([np.array(vols)[-10:], np.array(moms)])
    ref = np.concatenate([vref[-10:], mref])
    assert _pariscompare_l2(got, ref) < 1e-4


@pytest.mark.parametrize("rotation", [0, 1])
def test_curvature_sphere(capi, orc, rotation):
    """Tests/Curvature: 32^3 periodic, sphere R=0.32 at the centre,
    refinement 8; every mixed cell gets a curvature and kappa*Nx is within
    4e-2 (relative L2) of -2/R."""
    n = 32
    d = capi.make_desc((n, n, n), do_rotation=rotation)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [0.32], refinement=8)
    H = orc.get_all_heights(d, cvof, flag)
    kap, kf, mc = orc.get_all_curvatures(d, cvof, flag, H)
    mixed = orc.interior(d, flag) == 2
    k = orc.interior(d, kap)[mixed]
    assert np.all(k < 2e6)
    kn = k * n
    ex = -2.0 / 0.32
    rel = np.sqrt(np.mean((kn - ex) ** 2) / ex ** 2)
    assert rel < 4e-2
    assert mc[0] > 0.9 * mixed.sum()     # mostly nine-height curvatures


def test_heights_of_a_plane(capi, orc):
    """A plane interface z = 0.4375 + 0.3*h*...: the height in z of every
    pure cell of the stack equals the distance to the interface in cell units."""
    n = 16
    d = capi.make_desc((n, n, n))
    cvof = orc.zeros(d)
    zc = orc.grid_coords(d)["z"]
    # liquid (cvof=1) below z0, exact cell fractions
    z0 = 0.4 + 0.3 / n
    for kk in range(cvof.shape[0]):
        lo, hi = zc[kk] - 0.5 / n, zc[kk] + 0.5 / n
        cvof[kk] = np.clip((z0 - lo) * n, 0.0, 1.0)
    flag = np.where(cvof <= 0.0, 0, np.where(cvof >= 1.0, 1, 2)).astype(np.int32)
    H = orc.get_all_heights(d, cvof, flag)
    g = d.ng
    # liquid below, normal pointing up (+z): index 2*(3-1)+1 = 5 (0-based 4)
    for kk in range(g, g + n):
        hv = H[4, kk, g + 3, g + 5]
        if hv < 1e6:
            zc_cell = zc[kk]
            assert abs(hv - (z0 - zc_cell) * n) < 1e-12


def test_plic_identities(orc):
    rng = np.random.default_rng(0)
    for _ in range(300):
        m = rng.standard_normal(3)
        m /= np.abs(m).sum()
        c = rng.uniform(1e-6, 1 - 1e-6)
        a = orc.al3d(m, c)
        assert abs(orc.cc3d(m, a) - c) < 1e-12
        assert abs(orc.fl3d(m, a, [0, 0, 0], [1, 1, 1]) - c) < 1e-12
        # the two halves of the cube add up to the cell fraction
        h1 = orc.fl3d(m, a, [0, 0, 0], [0.5, 1, 1])
        h2 = orc.fl3d(m, a, [0.5, 0, 0], [0.5, 1, 1])
        assert abs(h1 + h2 - c) < 1e-12
        # the facet centroid lies on the plane
        xc = orc.area_centroid(m, c)
        assert abs(np.dot(m, xc) - a) < 1e-10
        assert orc.area3d(m, c) > 0


def test_mycs_of_a_plane(orc):
    """MYC returns the plane normal for a linear interface (|n|_1 = 1, pointing
    out of the reference phase)."""
    blk = np.zeros((3, 3, 3))
    for i in range(3):
        blk[i, :, :] = [1.0, 0.6, 0.0][i]
    m = orc.mycs(blk)
    assert abs(abs(m).sum() - 1) < 1e-12
    assert m[0] == pytest.approx(1.0) and abs(m[1]) < 1e-12 and abs(m[2]) < 1e-12
