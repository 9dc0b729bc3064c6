"""A projection problem shared by the tests that compare two forms of the
fused multigrid sweep: drops of density ratio 1000 from the level-set
initialisation and a random velocity field with zero normal velocity on the
walls."""
import numpy as np


def problem(capi, orc, workloads, n, bc, seed):
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


def assert_same_solve(p_a, r_a, p_b, r_b, pcg, mixed):
    """Two forms of the sweep smooth to the same bits, so a defect-correction
    solve (pcg 0) gives the same pressure to the bit.  With the CG outer loop
    the single fused sweep also forms r.z on its last finest-level pass (from
    the FP32 right-hand side it smooths, in the mixed cycle) where the other
    forms take a pass of their own, so there the CG scalars differ in their
    last bits: the same iteration count, and pressures equal to 1e-6 (mixed)
    or 1e-11 (FP64) of their largest value."""
    assert r_a.it == r_b.it
    if not pcg:
        assert r_a.rel_res == r_b.rel_res
        assert np.array_equal(p_a, p_b)
        return
    scale = float(np.abs(p_b).max())
    tol = 1e-6 if mixed else 1e-11
    assert abs(r_a.rel_res - r_b.rel_res) <= (1e-4 if mixed else 1e-9) * abs(r_b.rel_res)
    assert float(np.abs(p_a - p_b).max()) <= tol * scale
