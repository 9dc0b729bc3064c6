"""Full explicit Navier-Stokes steps on the GPU (ParisGpu.ns_step: the
order of the PARIS step loop, paris.f90:281-656) against the same steps on
the oracle: a drop in a closed box under surface tension and gravity.  The
pressure is solved by the reference multigrid on both sides.

Each step is checked from the same state on both sides: the states then
agree to the ulps of CUDA's versus glibc's transcendental functions in the
VOF and curvature geometry.  Run freely for several steps, those ulps can
flip a discrete PLIC decision (for example the choice between two nearly
equal candidate normals in a mixed cell), so the free run is checked to the
size of such a flip."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cvof", "u", "v", "w", "p")


def setup(capi, orc):
    n = 32   # the reference multigrid needs 2^n cells per direction (MGsolver.f90:43-46)
    d = capi.make_desc((n, n, n), bc="wall", rho1=1.0, rho2=10.0, mu1=0.01, mu2=0.1, sigma=0.05)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.45)], [0.2], refinement=8)
    st = {"cvof": cvof, "flag": flag, "u": orc.zeros(d), "v": orc.zeros(d), "w": orc.zeros(d), "p": orc.zeros(d)}
    return d, st


def upload(gpu, capi, st):
    gpu.upload(capi.F_CVOF, st["cvof"])
    gpu.upload(capi.F_VOF_FLAG, st["flag"])
    for f in ("u", "v", "w", "p"):
        gpu.upload(getattr(capi, "F_" + f.upper()), st[f])


def compare(capi, orc, d, out, ref, tol_c, tol_v, tol_p):
    g = d.ng
    inner = (slice(g, -g),) * 3
    assert np.abs(out["cvof"] - ref["cvof"]).max() <= tol_c
    vmax = max(np.abs(ref[c][inner]).max() for c in "uvw")
    assert vmax > 0
    for c in "uvw":
        assert np.abs(out[c] - ref[c]).max() <= tol_v * vmax, c
    pi, po = ref["p"][inner], out["p"][inner]
    assert np.abs((po - po.mean()) - (pi - pi.mean())).max() <= tol_p * np.abs(pi - pi.mean()).max()


DT, GRAV, MAXERR = 2e-3, (0.0, 0.0, -1.0), 1e-11


@pytest.mark.parametrize("scheme", [0, 1])
def test_each_step_from_the_same_state(gpu_lib, capi, runtime, orc, scheme):
    d, st = setup(capi, orc)
    solve = {"max_error": MAXERR, "maxit": 4000, "mode": capi.MG_REFERENCE}
    with runtime.ParisGpu(d) as gpu:
        for k in range(1, 6):
            upload(gpu, capi, st)
            gpu.ns_step(k, DT, scheme=scheme, gravity=GRAV, solve=solve)
            out = {f: gpu.download(getattr(capi, "F_" + f.upper())) for f in FIELDS}
            orc.ns_step(d, st, k, DT, scheme=scheme, gravity=GRAV, max_error=MAXERR, maxit=4000)
            compare(capi, orc, d, out, st, 1e-12, 1e-9, 1e-9)


def test_free_run_stays_on_the_oracle_trajectory(gpu_lib, capi, runtime, orc):
    d, st = setup(capi, orc)
    init = {k: v.copy() for k, v in st.items()}
    solve = {"max_error": MAXERR, "maxit": 4000, "mode": capi.MG_REFERENCE}
    for k in range(1, 6):
        orc.ns_step(d, st, k, DT, gravity=GRAV, max_error=MAXERR, maxit=4000)
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, init)
        for k in range(1, 6):
            gpu.ns_step(k, DT, gravity=GRAV, solve=solve)
        out = {f: gpu.download(getattr(capi, "F_" + f.upper())) for f in FIELDS}
    compare(capi, orc, d, out, st, 1e-6, 1e-4, 1e-4)
