"""Time-step control and flow statistics on the GPU against the oracle:
TimeStepSize and get_cfl_and_check bit for bit (a max is order-independent),
calcStats column by column.  The device sums the 25 columns in block
partials, the oracle in the reference's k,j,i loop order, so each column
agrees to the rounding of a reordered sum: 1e-12 of the sum of |term|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def state(capi, orc, bc, seed):
    n = 24
    d = capi.make_desc((n, n + 4, n - 4), bc=bc, rho1=1.2, rho2=1000.0, mu1=1.8e-5, mu2=1e-3,
                       length=(1.0, 28 / 24, 20 / 24))
    rng = np.random.default_rng(seed)
    cvof, flag, _ = orc.init_spheres(d, [(0.45, 0.6, 0.4), (0.7, 0.3, 0.45)], [0.2, 0.12], refinement=4)
    f = {"cvof": cvof, "flag": flag}
    for k in ("u", "v", "w", "p"):
        f[k] = rng.standard_normal(orc.shape(d))
    f["rho"] = 1.2 + (1000.0 - 1.2) * cvof
    f["mu"] = rng.uniform(1e-5, 1e-3, orc.shape(d))
    return d, f


FIELDS = {"u": "F_U", "v": "F_V", "w": "F_W", "rho": "F_RHO", "p": "F_P", "cvof": "F_CVOF", "mu": "F_MU",
          "flag": "F_VOF_FLAG"}


def upload(gpu, capi, f):
    for k, name in FIELDS.items():
        gpu.upload(getattr(capi, name), f[k])


def scale(d, ab):
    """The normalisations of calcStats applied to the sums of |term|."""
    s = ab.copy()
    V = d.xlength * d.ylength * d.zlength
    s[1:11] /= V
    s[0] /= d.xlength * d.zlength * 2.0
    return s


@pytest.mark.parametrize("bc", ["wall", "periodic"])
@pytest.mark.parametrize("flags", [0, 1, 6])
def test_calc_stats_follow_oracle(gpu_lib, capi, runtime, orc, bc, flags):
    d, f = state(capi, orc, bc, 5)
    o = capi.make_stats_opts(dpdx=(0.2, -0.1, 0.05), gravity=(0.0, -9.81, 0.3), buoyancy=3, rho_ave=400.0,
                             test_flags=flags)
    ref, ab = orc.calc_stats(d, f["u"], f["v"], f["w"], f["rho"], f["p"], f["cvof"], f["mu"], f["flag"], o)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, f)
        out = gpu.calc_stats(o)
    tol = 1e-12 * scale(d, ab)
    if flags & capi.STATS_RISING_BUBBLE:
        # columns 11 and 24 are divided by the phase volume afterwards
        tol[10] = 1e-12 * ab[10] / ab[9] + 1e-12
        tol[23] = 1e-12 * ab[23] / ref[9] + 1e-12
        tol[9] = 1e-12 * ab[9]
    bad = np.abs(out - ref) > tol
    assert not bad.any(), (np.nonzero(bad)[0] + 1, out[bad], ref[bad])
    assert out[16] == ref[16] and out[17] == ref[17]            # point values
    assert out[24] == ref[24] == np.count_nonzero(orc.interior(d, f["flag"]) == 2)
    assert out[18] > 0 and out[21] > 0 and out[22] > 0


def test_time_step_size_and_cfl_bitwise(gpu_lib, capi, runtime, orc):
    d, f = state(capi, orc, "wall", 7)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, f)
        for cfl, max_dt in ((0.5, 1.0), (0.25, 1e-3)):
            dt, vmax = gpu.time_step_size(cfl, max_dt)
            assert (dt, vmax) == orc.time_step_size(d, f["u"], f["v"], f["w"], cfl, max_dt)
        cfl = gpu.get_cfl_and_check(1e-3)
        assert orc.get_cfl_and_check(d, f["u"], f["v"], f["w"], 1e-3) == (0, cfl)
        with pytest.raises(runtime.ParisError) as e:
            gpu.get_cfl_and_check(1.0)
        assert e.value.status == capi.CFL_TOO_LARGE
        for k in ("u", "v", "w"):
            gpu.fill_field(getattr(capi, FIELDS[k]), 0.0)
        dt, vmax = gpu.time_step_size(0.5, 1e9)
        z = orc.zeros(d)
        assert vmax == 0.0 and (dt, vmax) == orc.time_step_size(d, z, z, z, 0.5, 1e9)   # the 1e-3 floor
