"""Static droplet (a full Navier-Stokes run, the droplet case of the
measurements): closed box of side 1, drop of radius 0.25 at the centre,
density ratio 1000, viscosity ratio 100, sigma = 1, liquid viscosity from a
Laplace number La = sigma rho_l D / mu_l^2 = 12000, at the capillary
time-step limit that PARIS checks its input against (paris.f90:3755-3773:
dx^3 rho1 / (dt^2 sigma) >= 2, phase 1 the gas), which also passes its
explicit viscous check (paris.f90:3750-3767: dx^2 rho1 / (dt mu1) >= 6).

At 128^3, 200 steps: the spurious currents (capillary number
max|u| mu_l / sigma), the curvature of the interface cells against the exact
-2/R (kappa is in grid units: kappa * n is compared), the Laplace pressure
jump 2 sigma / R, and the liquid volume, which the split VOF advection keeps
to round-off.  At 64^3 for 20 steps and at 128^3 for 10 steps: the same
run on the oracle, cvof, velocity and pressure compared."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R, RHO_L, RHO_G, SIGMA, LA = 0.25, 1000.0, 1.0, 1.0, 12000.0


def droplet(capi, n):
    mu_l = math.sqrt(SIGMA * RHO_L * 2 * R / LA)
    mu_g = mu_l / 100.0
    d = capi.make_desc((n, n, n), bc="wall", rho1=RHO_G, rho2=RHO_L, mu1=mu_g, mu2=mu_l, sigma=SIGMA)
    h = 1.0 / n
    dt = math.sqrt(h ** 3 * RHO_G / (2.0 * SIGMA))
    assert h ** 2 * RHO_G / (dt * mu_g) >= 6.0
    return d, dt, mu_l


def radius(d):
    n = d.nx
    c = (np.arange(n) + 0.5) / n - 0.5
    return np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)


def laplace_jump(d, p):
    """Mean pressure inside r < R - 3h minus outside r > R + 3h."""
    g, n = d.ng, d.nx
    r = radius(d)
    pi = p[g:-g, g:-g, g:-g]
    return pi[r < R - 3.0 / n].mean() - pi[r > R + 3.0 / n].mean()


def run(gpu, capi, runtime, steps, dt, solve=None):
    its = []
    for k in range(1, steps + 1):
        try:
            its.append(gpu.ns_step(k, dt, solve=solve).it)
        except runtime.ParisError as e:
            raise AssertionError(f"step {k}: {e}") from e
    return its


def test_static_droplet_128(gpu_lib, capi, runtime):
    n, steps = 128, 200
    d, dt, mu_l = droplet(capi, n)
    with runtime.ParisGpu(d) as gpu:
        gpu.init_spheres([(0.5, 0.5, 0.5)], [R], refinement=8)
        for f in (capi.F_U, capi.F_V, capi.F_W, capi.F_P):
            gpu.fill_field(f, 0.0)
        c0 = gpu.download(capi.F_CVOF)
        its = run(gpu, capi, runtime, steps, dt)
        u, v, w, p, c1 = (gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W, capi.F_P, capi.F_CVOF))
        gpu.get_all_heights()
        kap = gpu.get_all_curvatures()
        flag = gpu.download(capi.F_VOF_FLAG)
    g = d.ng
    inner = (slice(g, -g),) * 3
    umax = max(np.abs(a[inner]).max() for a in (u, v, w))
    ca = umax * mu_l / SIGMA
    k_in = kap[inner][flag[inner] == 2]
    assert np.all(k_in < 1e6)          # every mixed cell got a curvature
    ex = -2.0 / R
    kerr = np.sqrt(np.mean((k_in * n - ex) ** 2)) / abs(ex)
    dp = laplace_jump(d, p)
    perr = abs(dp - 2.0 * SIGMA / R) / (2.0 * SIGMA / R)
    vol0, vol1 = c0[inner].sum(), c1[inner].sum()
    print(f"\nstatic droplet {n}^3: dt {dt:.4e}, {steps} steps, t = {steps * dt:.4f}; solver iterations "
          f"{min(its)}..{max(its)}; max|u| {umax:.3e} (Ca {ca:.3e}); curvature error (rel. L2) {kerr:.3e} "
          f"over {k_in.size} cells; pressure jump {dp:.6f} (error {perr:.3e}); volume change "
          f"{abs(vol1 - vol0) / vol0:.3e} relative")
    assert ca < 1e-4
    assert kerr < 5e-3
    assert perr < 2e-2
    assert abs(vol1 - vol0) <= 1e-12 * vol0


@pytest.mark.parametrize("mode", ["reference", "mixed"])
def test_static_droplet_64_follows_oracle(gpu_lib, capi, runtime, orc, mode):
    n, steps = 64, 20
    d, dt, _ = droplet(capi, n)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [R], refinement=8)
    st = {"cvof": cvof, "flag": flag, "u": orc.zeros(d), "v": orc.zeros(d), "w": orc.zeros(d), "p": orc.zeros(d)}
    solve = {"max_error": 1e-11, "maxit": 4000, "mode": capi.MG_REFERENCE} if mode == "reference" else None
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_CVOF, st["cvof"])
        gpu.upload(capi.F_VOF_FLAG, st["flag"])
        for f in (capi.F_U, capi.F_V, capi.F_W, capi.F_P):
            gpu.fill_field(f, 0.0)
        run(gpu, capi, runtime, steps, dt, solve)
        out = {f: gpu.download(getattr(capi, "F_" + f.upper())) for f in ("cvof", "u", "v", "w", "p")}
    for k in range(1, steps + 1):
        orc.ns_step(d, st, k, dt, max_error=1e-11, maxit=4000)
    g = d.ng
    inner = (slice(g, -g),) * 3
    dc = np.abs(out["cvof"] - st["cvof"]).max()
    vmax = max(np.abs(st[c][inner]).max() for c in "uvw")
    du = max(np.abs(out[c] - st[c]).max() for c in "uvw") / vmax
    pi, po = st["p"][inner], out["p"][inner]
    dpr = np.abs((po - po.mean()) - (pi - pi.mean())).max() / (2.0 * SIGMA / R)
    print(f"\nstatic droplet {n}^3, {steps} steps, {mode} solver against the oracle: max |dcvof| {dc:.3e}, "
          f"max |du| / max|u| {du:.3e}, max |dp| / (2 sigma/R) {dpr:.3e}")
    tol = {"reference": (1e-12, 1e-9, 1e-10), "mixed": (1e-11, 1e-6, 1e-9)}[mode]
    assert dc <= tol[0]
    assert du <= tol[1]
    assert dpr <= tol[2]


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_static_droplet_128_follows_oracle(gpu_lib, capi, runtime, orc, mode):
    """The droplet at its stated size, 128^3, for 10 steps, each from the same
    state on both sides: the oracle's state after the previous step is
    uploaded, one step runs on each side, and cvof, velocity and pressure are
    compared.  The oracle solves with its FP64 restatement of the B200
    multigrid (flexible CG preconditioned by V(2,2) cycles) to
    ||r||/||b|| < 1e-10; the device with the same algorithm in FP64, or with
    FP32 cycles inside the FP64 loop (mixed).  Run free instead, the two
    sides part after a few steps where two candidate PLIC normals of a mixed
    cell tie to the last bit: CUDA's and glibc's pow/acos differ by an ulp,
    and one cell of cvof moves by 1.2e-9 (RMS 2.5e-12 over the box)."""
    n, steps = 128, 10
    d, dt, _ = droplet(capi, n)
    cvof, flag, _ = orc.init_spheres(d, [(0.5, 0.5, 0.5)], [R], refinement=8)
    st = {"cvof": cvof, "flag": flag, "u": orc.zeros(d), "v": orc.zeros(d), "w": orc.zeros(d), "p": orc.zeros(d)}
    solve = {"max_error": 0.0, "rel_tol": 1e-10, "maxit": 200, "pcg": 1,
             "mode": capi.MG_FP64 if mode == "fp64" else capi.MG_MIXED}
    g = d.ng
    inner = (slice(g, -g),) * 3
    rows = []
    with runtime.ParisGpu(d) as gpu:
        for k in range(1, steps + 1):
            gpu.upload(capi.F_CVOF, st["cvof"])
            gpu.upload(capi.F_VOF_FLAG, st["flag"])
            for c in "uvwp":
                gpu.upload(getattr(capi, "F_" + c.upper()), st[c])
            r = gpu.ns_step(k, dt, solve=solve)
            out = {f: gpu.download(getattr(capi, "F_" + f.upper())) for f in ("cvof", "u", "v", "w", "p")}
            it_ref = orc.ns_step(d, st, k, dt, solver="fast", rel_tol=1e-10, maxit=200)
            dc = np.abs(out["cvof"] - st["cvof"]).max()
            vmax = max(np.abs(st[c][inner]).max() for c in "uvw")
            du = max(np.abs(out[c] - st[c]).max() for c in "uvw") / vmax
            pi, po = st["p"][inner], out["p"][inner]
            dpr = np.abs((po - po.mean()) - (pi - pi.mean())).max() / (2.0 * SIGMA / R)
            rows.append((dc, du, dpr, r.it, it_ref, vmax))
    R_ = np.array(rows)
    print(f"\nstatic droplet {n}^3, {steps} steps from the same state, {mode} solver against the oracle: "
          f"max |dcvof| {R_[:, 0].max():.3e}, max |du| / max|u| {R_[:, 1].max():.3e} (max|u| up to "
          f"{R_[:, 5].max():.3e}), max |dp| / (2 sigma/R) {R_[:, 2].max():.3e}; iterations "
          f"{R_[:, 3].astype(int).tolist()} oracle {R_[:, 4].astype(int).tolist()}")
    # measured on a B200, both solvers: cvof 4.1e-11 (a PLIC normal chosen
    # between two candidates that tie to an ulp in one cell), velocity 1.5e-7 of
    # max |u| (1.1e-5), pressure 1.4e-10 of 2 sigma / R
    lim = {"fp64": (1e-10, 1e-6, 1e-9), "mixed": (1e-10, 1e-6, 1e-9)}[mode]
    assert R_[:, 0].max() <= lim[0]
    assert R_[:, 1].max() <= lim[1]
    assert R_[:, 2].max() <= lim[2]
