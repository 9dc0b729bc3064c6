"""SetVOFBC of the oracle (vofmodules.f90:1694-1825) for the 'jet' and
'90deg' conditions, checked cell by cell against the rules as the reference
writes them, and the "bad flag" stop of ls2vof_refined these faces cause."""
import numpy as np
import pytest


def _desc(capi, vofbc, n=8, jet=None):
    return capi.make_desc((n, n, n), bc="wall", vofbc=vofbc, jet=jet)


def test_90deg_copies_first_layer_only(capi, orc):
    V = capi.VOFBC_90DEG
    desc = _desc(capi, (V, V, V, V, V, V))
    rng = np.random.default_rng(0)
    c = rng.uniform(0.0, 1.0, orc.shape(desc))
    f = rng.integers(0, 3, orc.shape(desc)).astype(np.int32)
    c0 = c.copy()
    orc.setvofbc(desc, c, f)
    g, n = 2, 8
    # reference order: x-, y-, z-, x+, y+, z+ over the whole ghosted extent
    r = c0.copy()
    for o in range(6):
        d = o % 3
        ax = 2 - d                      # numpy axis of direction d
        lim = g if o < 3 else g + n - 1
        sgn = -1 if o < 3 else 1
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        src[ax] = lim
        dst[ax] = lim + sgn
        r[tuple(dst)] = r[tuple(src)]
    assert np.array_equal(c, r)
    # the second layers are untouched except where another face's first layer lies
    assert np.array_equal(c[g:-g, g:-g, 0], c0[g:-g, g:-g, 0])


@pytest.mark.parametrize("itype", [2, 3, 4, 5])
def test_jet_first_layer_is_inject(capi, orc, itype):
    desc = _desc(capi, (capi.VOFBC_JET, 0, 0, 0, 0, 0), n=16, jet=(itype, 0.5, 0.45, 0.3, 0.1))
    c = np.full(orc.shape(desc), 0.25)
    f = np.full(orc.shape(desc), 2, dtype=np.int32)
    orc.setvofbc(desc, c, f)
    h = 1.0 / 16
    yc = (np.arange(-2, 18) + 0.5) * h
    Z, Y = np.meshgrid(yc, yc, indexing="ij")
    yy, zz = Y - 0.5, Z - 0.45
    if itype in (2, 4):
        inj = yy * yy + zz * zz < 0.3 * 0.3
    elif itype == 3:
        inj = yy <= 0.3
    else:
        inj = (yy > 0.1) & (yy < 0.3)
    # x- first layer (numpy x index 1) over the y, z extent the later faces do not overwrite
    got = c[2:-2, 2:-2, 1]
    assert np.array_equal(got, inj[2:-2, 2:-2].astype(float))
    assert np.array_equal(f[2:-2, 2:-2, 1], inj[2:-2, 2:-2].astype(np.int32))
    # the second layer keeps its value
    assert np.all(c[2:-2, 2:-2, 0] == 0.25)


@pytest.mark.parametrize("cond", ["jet", "90deg"])
def test_levelset_init_stops_with_bad_flag(capi, orc, cond):
    code = capi.VOFBC_JET if cond == "jet" else capi.VOFBC_90DEG
    desc = _desc(capi, (code, 0, 0, 0, 0, 0), n=16, jet=(2, 0.5, 0.5, 0.2, 0.0))
    with pytest.raises(ValueError, match="bad flag"):
        orc.init_spheres(desc, [(0.5, 0.5, 0.5)], [0.25])
