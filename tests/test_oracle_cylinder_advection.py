"""The oracle's momentum-conserving step pinned to the reference's own
regression test Tests/CylinderAdvection: a 16 x 16 x 2 periodic box,
an elliptic cylinder (radius 0.1, excentricity (1, 0, 0), along z) of
density 1e5 in a fluid of density 1, both inviscid, advected by the uniform
velocity (0.01, 0.01, 0) for 3800 steps of dt = 0.1 with DoMOMCONS,
staggeredmom = T, LinInterp = F and the Weymouth-Yue sweeps.  The reference
prints the cvof of the mid plane with five significant digits
(tests/golden/cylinder_advection_cvof.txt, copied by make_fixtures.py); the
oracle must agree to those digits in every cell."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    with open(os.path.join(HERE, "golden", "cylinder_advection_cvof.txt")) as f:
        vals = [float(line) for line in f if line.strip() and not line.startswith("#")]
    return np.array(vals).reshape(16, 16)   # (i, j)


def test_cylinder_advection_matches_the_reference_output(capi, orc):
    d = capi.make_desc((16, 16, 2), length=(1.0, 1.0, 0.125), bc="periodic", rho1=1.0, rho2=1e5, mu1=0.0,
                       mu2=0.0, sigma=0.0)
    d.vof_advect = capi.ADVECT_WY
    cvof, flag, _ = orc.init_shapes(d, [(0.5, 0.5, 0.5)], [0.1], excentricity=(1.0, 0.0, 0.0), ipar=-3,
                                    refinement=8)
    st = {"cvof": cvof, "flag": flag, "u": np.full(orc.shape(d), 0.01), "v": np.full(orc.shape(d), 0.01),
          "w": orc.zeros(d), "p": orc.zeros(d)}
    for k in range(1, 3801):
        orc.ns_step(d, st, k, 0.1, max_error=1e-5, maxit=2000, momcons={"staggered": True, "lin_interp": False},
                    solver="fast")
    g = d.ng
    out = st["cvof"][g, g:-g, g:-g].T   # plane (ks+ke)/2 = ks, indexed (i, j)
    ref = golden()
    # half a unit of the fifth significant digit of each printed value; a
    # printed zero is an exact zero (E14.5 prints small values with their exponent)
    mag = np.floor(np.log10(np.where(ref == 0.0, 1.0, np.abs(ref))))
    tol = np.where(ref == 0.0, 1e-12, 0.5 * 10.0 ** (mag - 4) * (1.0 + 1e-6))
    err = np.abs(out - ref)
    assert (err <= tol).all(), (np.argwhere(err > tol)[:5], out[err > tol][:5], ref[err > tol][:5])
    # the uniform velocity stays uniform: the momentum flux is the velocity times the mass flux
    assert np.abs(st["u"] - 0.01).max() < 1e-14 and np.abs(st["v"] - 0.01).max() < 1e-14
    assert np.abs(st["w"]).max() == 0.0
