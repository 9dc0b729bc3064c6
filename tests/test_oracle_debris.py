"""Properties of the oracle's clean_debris (vofmodules.f90:2087-2234), no
GPU needed."""
import numpy as np
import pytest


def sphere_with_specks(capi, orc, bc="periodic", n=24, seed=0):
    d = capi.make_desc((n, n, n), bc=bc)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [0.25], refinement=4)
    g = d.ng
    rng = np.random.default_rng(seed)
    # specks: small fractions deep in the gas, small holes deep in the liquid
    gas = [(g + 1, g + 1, g + 1), (g + n - 3, g + 2, g + n - 4)]
    liq = [(g + n // 2, g + n // 2, g + n // 2)]
    for k, j, i in gas:
        cvof[k, j, i] = rng.uniform(0.01, 0.05)
    for k, j, i in liq:
        cvof[k, j, i] = 1.0 - rng.uniform(0.01, 0.05)
    orc.fill_ghosts(d, cvof)
    orc.flags_clip(d, cvof, flag)
    return d, cvof, flag, gas, liq


@pytest.mark.parametrize("method", [1, 2])
def test_specks_removed_interface_kept(capi, orc, method):
    d, cvof, flag, gas, liq = sphere_with_specks(capi, orc)
    before = cvof.copy()
    assert orc.clean_debris(d, cvof, flag, method, 2) == 1
    for k, j, i in gas:
        assert cvof[k, j, i] == 0.0
    for k, j, i in liq:
        assert cvof[k, j, i] == 1.0
    g = d.ng
    inner = (slice(g, -g),) * 3
    changed = np.argwhere(orc.interior(d, cvof) != orc.interior(d, before))
    assert len(changed) == len(gas) + len(liq)   # nothing else moves


def test_method3_isolated_mixed_cell_and_sweep_count(capi, orc):
    d, cvof, flag, gas, liq = sphere_with_specks(capi, orc)
    n_sweeps = orc.clean_debris(d, cvof, flag, 3, 2)
    assert n_sweeps == 11                  # the count of cleaned cells never resets
    for k, j, i in gas:
        assert cvof[k, j, i] == 0.0 and flag[k, j, i] == 0
    for k, j, i in liq:
        assert cvof[k, j, i] == 1.0 and flag[k, j, i] == 1
    # a smooth interface (every mixed cell has many mixed neighbours) is left
    # alone, in one sweep
    d2 = capi.make_desc((24, 24, 24))
    c2, f2, _ = orc.init_spheres(d2, [(0.5, 0.5, 0.5)], [0.3], refinement=4)
    c0 = c2.copy()
    assert orc.clean_debris(d2, c2, f2, 3, 2) == 1
    assert np.array_equal(c2, c0)


def test_two_dimensional_case_has_no_z_neighbourhood(capi, orc):
    """Nz = 2 (the reference's 2-D runs): the neighbourhood has no z extent,
    so a speck is judged by its own plane only."""
    d = capi.make_desc((16, 16, 2))
    c = orc.zeros(d)
    f = orc.zeros(d, np.int32)
    g = d.ng
    c[g:-g, g:-g, g:-g] = 1.0
    c[g, g + 8, g + 8] = 0.97        # a near-full cell in the liquid plane
    c[g + 1, :, :] = 0.0             # the other plane is gas
    orc.fill_ghosts(d, c)
    orc.flags_clip(d, c, f)
    orc.clean_debris(d, c, f, 1, 2)
    assert c[g, g + 8, g + 8] == 1.0
