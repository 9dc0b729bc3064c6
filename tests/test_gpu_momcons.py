"""The momentum-conserving VOF sweeps (vofandmomsweepsstaggered, DoMOMCONS)
on the device against the oracle, through the C-ABI: staggered and centred
control volumes, CIAM and Weymouth-Yue sweeps, LinInterp, the slope limiters
of interpole3, periodic boxes and walls (resting and moving).  Two calls in
a row share the persistent momentum array, as in the reference, and each is
compared.  The PLIC geometry (AL3D) uses cube roots and trigonometric
functions, so results agree to their rounding, not bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = (20, 16, 24)   # h = 1/16
CONFIGS = [("stg", "CIAM", False), ("stg", "CIAM", True), ("stg", "WY", False), ("stg", "WY", True),
           ("cen", "CIAM", False), ("cen", "WY", False)]
SCHEMES = ["QUICK", "ENO", "SUPERBEE", "WENO"]


def setup_state(capi, orc, cfg, bc, seed):
    kind, advect, lin = cfg
    h = 1.0 / 16
    d = capi.make_desc(N, length=tuple(n * h for n in N), bc=bc, rho1=1.0, rho2=20.0)
    d.vof_advect = capi.ADVECT_CIAM if advect == "CIAM" else capi.ADVECT_WY
    rng = np.random.default_rng(seed)
    cen = np.column_stack([rng.uniform(0.3, 0.9, 4) * N[0] * h, rng.uniform(0.3, 0.7, 4) * N[1] * h,
                           rng.uniform(0.3, 1.2, 4) * N[2] * h])
    cvof, flag, _ = orc.init_spheres(d, cen, rng.uniform(0.12, 0.22, 4), refinement=4)
    st = {"cvof": cvof, "flag": flag}
    for f in ("u", "v", "w"):
        a = 0.3 * rng.standard_normal(orc.shape(d))
        orc.fill_ghosts(d, a)
        st[f] = a
    if bc != "periodic":
        orc.set_velocity_bc(d, st["u"], st["v"], st["w"], None)
    for f in ("du", "dv", "dw"):
        st[f] = rng.standard_normal(orc.shape(d))
    st["mom"] = orc.zeros(d)
    dt = 0.4 * h / max(np.abs(st[f]).max() for f in ("u", "v", "w"))
    return d, st, dt


def upload(gpu, capi, st):
    for f in ("cvof", "u", "v", "w", "du", "dv", "dw"):
        gpu.upload(getattr(capi, "F_" + f.upper()), st[f])
    gpu.upload(capi.F_VOF_FLAG, st["flag"])


def compare(d, capi, gpu, st, tag):
    """Interior to tol of the interior's largest value; every element
    (ghosts included, where a wall line may hold a large power or a NaN)
    to 1e-9 relative, NaN where the oracle has NaN."""
    g = d.ng
    inner = (slice(g, -g),) * 3
    for f, tol in (("du", 1e-9), ("dv", 1e-9), ("dw", 1e-9), ("mom", 1e-11)):
        out = gpu.download(capi.F_MOMENTUM if f == "mom" else getattr(capi, "F_" + f.upper()))
        ref = st[f]
        scale = np.abs(ref[inner]).max()
        di = np.abs(out[inner] - ref[inner])
        assert di.max() <= tol * scale, (tag, f, di.max(), scale, np.unravel_index(di.argmax(), di.shape))
        ok = np.isclose(out, ref, rtol=1e-9, atol=tol * scale, equal_nan=True)
        assert ok.all(), (tag, f, np.argwhere(~ok)[:5], out[~ok][:5], ref[~ok][:5])


def run_case(capi, runtime, orc, cfg, bc, scheme, wall_vel=None, seed=11):
    d, st, dt = setup_state(capi, orc, cfg, bc, seed)
    kind, _, lin = cfg
    sc = getattr(capi, "CONV_" + scheme)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, st)
        for tswap in (1, 2):
            gpu.vof_mom_sweeps(tswap, dt, staggered=kind == "stg", lin_interp=lin, scheme=sc, wall_vel=wall_vel)
            orc.vof_mom_sweeps(d, tswap, dt, st["cvof"], st["flag"], st["u"], st["v"], st["w"], st["du"], st["dv"],
                               st["dw"], st["mom"], staggered=kind == "stg", lin_interp=lin, scheme=sc,
                               wall_vel=wall_vel)
            compare(d, capi, gpu, st, (cfg, bc, scheme, tswap))
        # the volume fraction and its flags are read only
        assert np.array_equal(gpu.download(capi.F_CVOF), st["cvof"])


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("cfg", CONFIGS, ids=["-".join(str(x) for x in c) for c in CONFIGS])
def test_momcons_periodic(gpu_lib, capi, runtime, orc, cfg, scheme):
    run_case(capi, runtime, orc, cfg, "periodic", scheme)


@pytest.mark.parametrize("cfg", CONFIGS, ids=["-".join(str(x) for x in c) for c in CONFIGS])
def test_momcons_walls(gpu_lib, capi, runtime, orc, cfg):
    run_case(capi, runtime, orc, cfg, "wall", "QUICK")


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[3]], ids=["stg-CIAM-lin", "stg-WY-lin"])
def test_momcons_moving_walls_mixed_boundaries(gpu_lib, capi, runtime, orc, cfg):
    """Walls in y and z (moving), periodic in x, a limiter scheme."""
    wv = np.zeros((6, 3))
    wv[2, 0], wv[3, 0], wv[4, 0], wv[5, 0] = 0.2, -0.1, 0.05, 0.3
    bc = [capi.BC_PERIODIC, capi.BC_WALL, capi.BC_WALL, capi.BC_PERIODIC, capi.BC_WALL, capi.BC_WALL]
    run_case(capi, runtime, orc, cfg, bc, "SUPERBEE", wall_vel=wv)


def test_momcons_rejects_unsupported_boundaries(gpu_lib, capi, runtime, orc):
    d, st, dt = setup_state(capi, orc, CONFIGS[0], "periodic", 1)
    for f in (1, 4):
        d.bdry_cond[f] = capi.BC_SHEAR
        d.vofbdry_cond[f] = capi.VOFBC_DRY
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, st)
        with pytest.raises(runtime.ParisError):
            gpu.vof_mom_sweeps(1, dt)
