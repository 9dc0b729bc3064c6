"""Parity of the pressure projection on the GPU against the FP64 oracle.

SetupPoisson and project_velocity must match bit for bit (same operation
order, no FMA); the reference multigrid must reproduce the oracle's iterates;
the B200 multigrid (FP64 and mixed) must converge to the oracle's solution
within the residual tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def drop_problem(capi, orc, workloads, n, bc="periodic", ndrops=6, seed=0, ratio=1000.0):
    desc = capi.make_desc((n, n, n), bc=bc, rho1=1.0, rho2=ratio)
    cen, rad = workloads.drop_layout(ndrops, rmin=0.1, rmax=0.2, seed=seed, h=1.0 / n)
    cvof, flag, _ = orc.init_spheres(desc, cen, rad, refinement=4)
    rho = orc.linfunc(desc, cvof, desc.rho1, desc.rho2, capi.MEAN_ARITH)
    rng = np.random.default_rng(seed + 7)
    vel = []
    for _ in range(3):
        f = orc.zeros(desc)
        orc.interior(desc, f)[...] = rng.standard_normal((n, n, n))
        if bc == "periodic":
            orc.fill_ghosts(desc, f)
        vel.append(f)
    if bc == "wall":
        # no flow through the walls: u(is-1) = u(ie) = 0 etc.
        g = desc.ng
        vel[0][:, :, g - 1] = 0.0
        vel[0][:, :, g + n - 1] = 0.0
        vel[1][:, g - 1, :] = 0.0
        vel[1][:, g + n - 1, :] = 0.0
        vel[2][g - 1, :, :] = 0.0
        vel[2][g + n - 1, :, :] = 0.0
    return desc, cvof, rho, vel


def upload_state(gpu, capi, cvof, rho, vel, p=None):
    gpu.upload(capi.F_CVOF, cvof)
    gpu.upload(capi.F_RHO, rho)
    for f, a in zip((capi.F_U, capi.F_V, capi.F_W), vel):
        gpu.upload(f, a)
    gpu.upload(capi.F_P, p if p is not None else np.zeros_like(cvof))


@pytest.mark.parametrize("n", [16, 24])
@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_setup_poisson_bitwise(gpu_lib, capi, runtime, orc, workloads, bc, n):
    """A (all eight components, as the reference stores them) equals the
    oracle's bit for bit: at 16^3 the spacing is a power of two and the
    divergence multiplies by its exact reciprocal, at 24^3 it divides."""
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc=bc)
    dt = 1e-3
    st, A_ref = orc.setup_poisson(desc, *vel, rho, dt)
    assert st == 0
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(dt)
        A = gpu.download(capi.F_A)
    assert np.array_equal(A, A_ref)


@pytest.mark.parametrize("n", [16, 24])
@pytest.mark.parametrize("case", ["nan_rho", "nan_u", "heavy", "negative_rho"])
def test_setup_poisson_checks(gpu_lib, capi, runtime, orc, workloads, case, n):
    """SetupPoisson refuses what the reference's checks refuse: a NaN in A,
    or A7 below 1e-50 outside a solid (a density of 1e60 everywhere, or a
    negative density that makes the coefficients of a cell negative)."""
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc="wall")
    g = desc.ng
    c = (g + n // 2, g + n // 3, g + n // 4)
    if case == "nan_rho":
        rho[c] = np.nan
    elif case == "nan_u":
        vel[0][c] = np.nan
    elif case == "heavy":
        rho[...] = 1e60
    else:
        rho[c] = -3.0 * np.abs(rho).max()
    dt = 1e-3
    st, _ = orc.setup_poisson(desc, *vel, rho, dt)
    assert st == capi.SETUP_ERROR
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        with pytest.raises(runtime.ParisError) as e:
            gpu.setup_poisson(dt)
        assert e.value.status == capi.SETUP_ERROR


def test_linfunc_bitwise(gpu_lib, capi, runtime, orc, workloads):
    desc, cvof, rho_ref, vel = drop_problem(capi, orc, workloads, 16)
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.linfunc(capi.F_RHO)
        rho = gpu.download(capi.F_RHO)
    assert np.array_equal(rho, rho_ref)


@pytest.mark.parametrize("nfilter", [0, 1])
@pytest.mark.parametrize("mean", [101, 102])
@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_linfunc_means_and_filter(gpu_lib, capi, runtime, orc, workloads, nfilter, mean, bc):
    """linfunc (vofmodules.f90:171-218) for rho and mu with the arithmetic and
    the harmonic mean, unfiltered and with the 27-point filter (nfilter = 1),
    bit for bit against the oracle, ghosts included."""
    n = 16
    desc = capi.make_desc((n, n, n), bc=bc, rho1=1.0, rho2=1000.0, mu1=1.8e-5, mu2=1e-3, nfilter=nfilter,
                          dens_mean=mean, visc_mean=203 - mean)
    cen, rad = workloads.drop_layout(6, rmin=0.1, rmax=0.2, seed=2, h=1.0 / n)
    cvof, flag, _ = orc.init_spheres(desc, cen, rad, refinement=4)
    rho_ref = orc.linfunc(desc, cvof, desc.rho1, desc.rho2, mean)
    mu_ref = orc.linfunc(desc, cvof, desc.mu1, desc.mu2, 203 - mean)
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.linfunc(capi.F_RHO)
        gpu.linfunc(capi.F_MU)
        rho = gpu.download(capi.F_RHO)
        mu = gpu.download(capi.F_MU)
    assert np.array_equal(rho, rho_ref)
    assert np.array_equal(mu, mu_ref)


def test_poissonmg_known_answer(gpu_lib, capi, runtime, orc):
    """Tests/PoissonMG: 32x16x16 periodic, XLENGTH=2, 20 V-cycles; residual
    < 1e-8 and L1 error < 0.1 (Tests/PoissonMG/run.sh:13), same iterates as
    the oracle."""
    desc = capi.make_desc((32, 16, 16), length=(2.0, 1.0, 1.0), rho1=1.0, rho2=1e5)
    rho = orc.zeros(desc) + 1.0
    A = orc.setup_testmg(desc, rho)
    p_ref = orc.zeros(desc)
    st, it, tres_ref, hist = orc.new_solver_mg(desc, A, p_ref, 1e-300, beta=1.0, maxit=20, norm=2)
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_RHO, rho)
        gpu.setup_test_mg()
        A_gpu = gpu.download(capi.F_A)
        # A1..A7 bit for bit; the sin() of the right-hand side may differ by
        # an ulp between the device and glibc
        assert np.array_equal(A_gpu[:7], A[:7])
        assert np.abs(A_gpu[7] - A[7]).max() <= 1e-14 * np.abs(A[7]).max()
        gpu.upload(capi.F_P, orc.zeros(desc))
        with pytest.warns(UserWarning):
            r = gpu.new_solver(1e-300, beta=1.0, maxit=20, norm=2, mode=capi.MG_REFERENCE)
        p = gpu.download(capi.F_P)
        err = gpu.mg_test_err()
    assert r.it == 21
    assert r.res < 1e-8 and err < 0.1
    assert abs(r.res - tres_ref) <= 1e-6 * tres_ref
    assert np.abs(orc.interior(desc, p) - orc.interior(desc, p_ref)).max() <= 1e-12


@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_reference_mg_iterates(gpu_lib, capi, runtime, orc, workloads, bc):
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, 16, bc=bc)
    dt = 1e-3
    st, A = orc.setup_poisson(desc, *vel, rho, dt)
    p_ref = orc.zeros(desc)
    orc.new_solver_mg(desc, A, p_ref, 1e-300, beta=1.0, maxit=5, norm=2)
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(dt)
        with pytest.warns(UserWarning):
            gpu.new_solver(1e-300, beta=1.0, maxit=5, norm=2, mode=capi.MG_REFERENCE)
        p = gpu.download(capi.F_P)
    scale = np.abs(orc.interior(desc, p_ref)).max()
    assert np.abs(orc.interior(desc, p) - orc.interior(desc, p_ref)).max() <= 1e-12 * scale


@pytest.mark.parametrize("mode,pcg", [(2, 0), (1, 0), (2, 1), (1, 1)])
@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_fast_mg_converges_to_oracle(gpu_lib, capi, runtime, orc, workloads, mode, pcg, bc):
    """The B200 multigrid reaches ||r||/||b|| < 1e-10; its pressure agrees with
    the oracle's FP64 solution of the same system (up to the constant of the
    singular periodic/closed problem) to the tolerance amplified by the
    condition of the operator."""
    n = 32
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc=bc)
    dt = 1e-3
    st, A = orc.setup_poisson(desc, *vel, rho, dt)
    p_ref, it_ref, _ = orc.fastmg_solve(desc, A, np.zeros((n, n, n)), 1e-12, maxit=100, mixed=False, pcg=True)
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(dt)
        r = gpu.new_solver(0.0, maxit=60, mode=mode, rel_tol=1e-10, pcg=pcg)
        p = orc.interior(desc, gpu.download(capi.F_P))
        assert r.rel_res < 1e-10
        assert r.it <= 25
        # the residual computed independently in FP64 on the device
        L1, L2, Linf = gpu.calc_residuals()
    b = A[7]
    assert L2 * np.sqrt(b.size) / np.sqrt((b ** 2).sum()) < 2e-10
    d = (p - p.mean()) - (p_ref - p_ref.mean())
    assert np.abs(d).max() <= 1e-7 * np.abs(p_ref - p_ref.mean()).max()


@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_project_velocity_bitwise(gpu_lib, capi, runtime, orc, workloads, bc):
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, 16, bc=bc)
    dt = 1e-3
    rng = np.random.default_rng(5)
    p = orc.zeros(desc)
    orc.interior(desc, p)[...] = rng.standard_normal((16, 16, 16))
    if bc == "periodic":
        orc.fill_ghosts(desc, p)
    ref = [v.copy() for v in vel]
    orc.project_velocity(desc, *ref, p, rho, dt)
    for v in ref:
        if bc == "periodic":
            orc.fill_ghosts(desc, v)
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel, p)
        gpu.project_velocity(dt)
        out = [gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W)]
    for a, b in zip(out, ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("beta,bcoarse,nuc,cf,ct", [(1.0, 0.0, 0, 0, 0), (1.1, 0.0, 0, 0, 0), (1.1, 0.0, 4, 1, 0),
                                                     (1.1, 0.0, 3, 2, 0), (1.1, 0.0, 4, 1, 2), (1.1, 1.25, 4, 1, 2)])
@pytest.mark.parametrize("bc,n", [("periodic", 64), ("wall", 64), ("periodic", 128)])
def test_fast_mg_fused_levels_follow_oracle(gpu_lib, capi, runtime, orc, workloads, bc, n, beta, bcoarse, nuc, cf,
                                            ct):
    """From 32^3 up the finest levels run the fused red-black sweep; the FP64
    V-cycle must follow the oracle's FP64 cycle: the same number of PCG
    iterations to 1e-10 and the same final residual to rounding; the mixed
    cycle the oracle's FP32 cycle within one iteration.  beta is the
    smoother's relaxation factor (1: Gauss-Seidel, 1.1: over-relaxed), bcoarse
    (when > 0) its factor on the levels below the finest; nuc sweeps each way
    on the levels cf..ct (ct 0: down to the coarsest; nuc 0: two, as on the
    finest)."""
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc=bc, ndrops=12)
    dt = 1e-3
    st, A = orc.setup_poisson(desc, *vel, rho, dt)
    p_ref, it_ref, hist = orc.fastmg_solve(desc, A, np.zeros((n, n, n)), 1e-10, maxit=60, mixed=False, pcg=True,
                                           omega=beta, nu_coarse=nuc, coarse_from=cf, coarse_to=ct,
                                           omega_coarse=bcoarse)
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(dt)
        r = gpu.new_solver(0.0, beta=beta, maxit=60, mode=capi.MG_FP64, rel_tol=1e-10, pcg=1, nu_coarse=nuc,
                           coarse_from=cf, coarse_to=ct, beta_coarse=bcoarse)
        p = orc.interior(desc, gpu.download(capi.F_P))
        gpu.fill_field(capi.F_P, 0.0)
        rm = gpu.new_solver(0.0, beta=beta, maxit=60, mode=capi.MG_MIXED, rel_tol=1e-10, pcg=1, nu_coarse=nuc,
                            coarse_from=cf, coarse_to=ct, beta_coarse=bcoarse)
    assert r.it == it_ref
    assert abs(r.rel_res - hist[-1]) <= 1e-6 * hist[-1]
    d = (p - p.mean()) - (p_ref - p_ref.mean())
    assert np.abs(d).max() <= 1e-9 * np.abs(p_ref - p_ref.mean()).max()
    assert rm.rel_res < 1e-10 and rm.it <= it_ref + 2
    _, itm_ref, _ = orc.fastmg_solve(desc, A, np.zeros((n, n, n)), 1e-10, maxit=60, mixed=True, pcg=True,
                                     omega=beta, nu_coarse=nuc, coarse_from=cf, coarse_to=ct, omega_coarse=bcoarse)
    assert abs(rm.it - itm_ref) <= 1


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_warm_start_with_a_large_constant(gpu_lib, capi, runtime, orc, workloads, mode):
    """Walls leave the pressure equation singular.  A warm start carrying a
    large constant (the hydrostatic level a previous step leaves in p) must
    converge like a cold start: the solver takes the mean of the initial
    guess out for the solve and puts it back, so the returned p keeps the
    caller's level (up to the mean of the correction)."""
    n = 128
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc="wall", ndrops=12)
    m = capi.MG_FP64 if mode == "fp64" else capi.MG_MIXED
    dt = 1e-3
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(dt)
        cold = gpu.new_solver(0.0, maxit=60, mode=m, rel_tol=1e-10, pcg=1)
        p = gpu.download(capi.F_P)
        rng = np.random.default_rng(3)
        g = desc.ng
        warm = p + 1e5
        orc.interior(desc, warm)[...] += 1e-3 * np.abs(p).max() * rng.standard_normal((n, n, n))
        gpu.upload(capi.F_P, warm)
        r = gpu.new_solver(0.0, maxit=60, mode=m, rel_tol=1e-10, pcg=1)
        pw = gpu.download(capi.F_P)
    assert cold.rel_res < 1e-10 and r.rel_res < 1e-10 and r.it <= cold.it
    wi = orc.interior(desc, warm)
    # the level: the warm start's mean plus the small mean of the solver's correction
    assert abs(orc.interior(desc, pw).mean() - wi.mean()) <= 1e-6 * abs(wi.mean())
    d = orc.interior(desc, pw) - orc.interior(desc, p)
    assert np.abs(d - d.mean()).max() <= 1e-8 * np.abs(p).max()


def test_fast_mg_rejects_negative_sweep_options(gpu_lib, capi, runtime, orc, workloads):
    """nu_coarse, coarse_from and coarse_to must not be negative: the solver
    refuses them with PARIS_BAD_ARGS before touching p."""
    n = 32
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, n, bc="periodic", ndrops=4)
    with runtime.ParisGpu(desc) as gpu:
        upload_state(gpu, capi, cvof, rho, vel)
        gpu.setup_poisson(1e-3)
        for bad in ({"nu_coarse": -1}, {"coarse_from": -1}, {"coarse_to": -1}):
            with pytest.raises(runtime.ParisError) as e:
                gpu.new_solver(0.0, maxit=5, mode=capi.MG_MIXED, rel_tol=1e-10, pcg=1, **bad)
            assert e.value.status == capi.BAD_ARGS
