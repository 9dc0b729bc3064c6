"""The projection adjoint on the GPU (paris_projection_adjoint) against the
CPU oracle's adjoint, against central finite differences of the GPU forward
(SetupPoisson + NewSolver + project_velocity) and through a
torch.autograd.Function wrapper checked by torch.autograd.gradcheck.

Loss L = sum over the faces project_velocity updates of w * u_proj, w and u*
standard normal; the parameters are u* and the face coefficients
B = 2/(rho_L + rho_R), whose gradient is checked through rho by the chain
rule dB_f/drho = -B_f^2/2 (the forward takes rho)."""
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORACLE_RTOL = 1e-8     # GPU adjoint vs oracle adjoint (both FP64, solves to 1e-12 / 1e-15)
FD_RTOL = 1e-6         # adjoint vs central differences, eps = 1e-6 (relative for rho), per entry
FD_FLOOR = 0.2         # entries checked per entry: |gradient| >= FD_FLOOR * the largest sampled one


def faces_of(orc, d):
    return [orc.updated_faces(d, k) for k in range(3)]


def make_case(capi, orc, n, bc, seed, layout):
    d = capi.make_desc((n, n, n), bc=bc, rho1=1.0, rho2=1000.0)
    rng = np.random.default_rng(seed)
    m = faces_of(orc, d)
    us = [rng.standard_normal(orc.shape(d)) for _ in range(3)]
    w = [rng.standard_normal(orc.shape(d)) for _ in range(3)]
    for a, b, mk in zip(us, w, m):
        a[~mk] = 0.0
        b[~mk] = 0.0
        orc.fill_ghosts(d, a)
    cen, rad = layout
    return d, us, w, m, cen, rad


def gpu_forward(gpu, capi, dt, us, p0=None, rel_tol=1e-14, maxit=60, project=True):
    for f, a in zip((capi.F_U, capi.F_V, capi.F_W), us):
        gpu.upload(f, a)
    gpu.setup_poisson(dt)
    if p0 is None:
        gpu.fill_field(capi.F_P, 0.0)
    else:
        gpu.upload(capi.F_P, p0)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        gpu.new_solver(0.0, maxit=maxit, mode=capi.MG_FP64, rel_tol=rel_tol, pcg=1)
    if not project:
        return None
    gpu.project_velocity(dt)
    return [gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W)]


def loss_diff(w, m, u1, u2):
    return sum(float((a * (b - c))[mk].sum()) for a, b, c, mk in zip(w, u1, u2, m))


def rho_chain(orc, d, rho, gb):
    """dL/drho on the interior from dL/dB (periodic directions)."""
    r = orc.interior(d, rho)
    out = np.zeros_like(r)
    for k, ax in enumerate((2, 1, 0)):
        B = 2.0 / (r + np.roll(r, -1, axis=ax))
        c = -0.5 * B * B * orc.interior(d, gb[k])
        out += c + np.roll(c, 1, axis=ax)
    return out


@pytest.mark.parametrize("bc,n", [("periodic", 16), ("wall", 16), ("periodic", 32), ("wall", 32)])
def test_adjoint_matches_oracle(gpu_lib, capi, runtime, orc, bc, n):
    layout = ([(0.4, 0.45, 0.5), (0.7, 0.3, 0.6), (0.2, 0.75, 0.3)], [0.2, 0.15, 0.12])
    d, us, w, m, cen, rad = make_case(capi, orc, n, bc, 3, layout)
    dt = 0.25 / n
    with runtime.ParisGpu(d) as gpu:
        gpu.init_spheres(cen, rad, refinement=4)
        gpu.linfunc(capi.F_RHO)
        rho = gpu.download(capi.F_RHO)
        gpu_forward(gpu, capi, dt, us)
        p = gpu.download(capi.F_P)
        gs, gb = gpu.projection_adjoint(dt, w)
    B = orc.face_B(d, rho)
    gs_ref, gb_ref, _ = orc.projection_adjoint(d, dt, B, p, w)
    for a, b, mk in zip(gs, gs_ref, m):
        assert np.all(a[~mk] == 0.0)
        assert np.abs(a - b).max() <= ORACLE_RTOL * np.abs(b).max()
    for a, b, mk in zip(gb, gb_ref, m):
        assert np.all(a[~mk] == 0.0)
        assert np.abs(a - b).max() <= ORACLE_RTOL * np.abs(b).max()


def fd_forward(gpu, capi, dt, us, p0):
    """A forward for differencing, from the unperturbed pressure: FP64 PCG to
    ||r||/||b|| < 1e-15, then four FP64 defect-correction cycles that take the
    true residual b - A p to its FP64 floor (the base solve's 1e-14 would
    leave ~1e-5 of the response to a 1e-6 perturbation unresolved at 128^3;
    CG itself is not run below the floor, where its recurrences drift)."""
    gpu_forward(gpu, capi, dt, us, p0, rel_tol=1e-15, maxit=60, project=False)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        gpu.new_solver(0.0, maxit=4, mode=capi.MG_FP64, rel_tol=1e-300, pcg=0)
    gpu.project_velocity(dt)
    return [gpu.download(f) for f in (capi.F_U, capi.F_V, capi.F_W)]


def test_adjoint_finite_differences_128(gpu_lib, capi, runtime, orc):
    """128^3 periodic, the 64-drop layout of the 256^3 workload rescaled,
    density ratio 1000; 120 u* entries and 80 rho entries (each rho entry
    tests the six dL/dB of its faces)."""
    n = 128
    wl = runtime_workloads()
    cen, rad = wl.drop_layout(64, rmin=0.03, rmax=0.08, seed=0, h=1.0 / n)
    d, us, w, m, _, _ = make_case(capi, orc, n, "periodic", 11, (cen, rad))
    dt = 0.25 / n
    rng = np.random.default_rng(12)
    errs_u, errs_r = [], []
    with runtime.ParisGpu(d) as gpu:
        gpu.init_spheres(cen, rad, refinement=4)
        gpu.linfunc(capi.F_RHO)
        rho = gpu.download(capi.F_RHO)
        u0 = gpu_forward(gpu, capi, dt, us)
        p0 = gpu.download(capi.F_P)
        gs, gb = gpu.projection_adjoint(dt, w)
        g = d.ng
        for _ in range(120):
            k = int(rng.integers(3))
            q = tuple(int(rng.integers(g, g + n)) for _ in range(3))
            eps = 1e-6
            up = [a.copy() for a in us]
            up[k][q] += eps
            orc.fill_ghosts(d, up[k])
            um = [a.copy() for a in us]
            um[k][q] -= eps
            orc.fill_ghosts(d, um[k])
            fd = loss_diff(w, m, fd_forward(gpu, capi, dt, up, p0), fd_forward(gpu, capi, dt, um, p0)) / (2 * eps)
            errs_u.append((fd, gs[k][q]))
        for f, a in zip((capi.F_U, capi.F_V, capi.F_W), us):
            gpu.upload(f, a)
        gr = rho_chain(orc, d, rho, gb)
        for _ in range(80):
            q = tuple(int(rng.integers(0, n)) for _ in range(3))
            qq = tuple(c + g for c in q)
            eps = 1e-6 * rho[qq]
            res = []
            for s in (1.0, -1.0):
                r1 = rho.copy()
                r1[qq] += s * eps
                orc.fill_ghosts(d, r1)
                gpu.upload(capi.F_RHO, r1)
                res.append(fd_forward(gpu, capi, dt, us, p0))
            fd = loss_diff(w, m, res[0], res[1]) / (2 * eps)
            errs_r.append((fd, gr[q]))
    # per entry: |fd - ad| / |ad| over the entries whose |ad| is at least
    # FD_FLOOR of the largest sampled one.  The central difference carries an
    # absolute error (rounding of the forward solves over eps), so entries far
    # below the largest one are checked against that absolute level instead.
    for name, e in (("u*", np.array(errs_u)), ("rho", np.array(errs_r))):
        fd, ad = e[:, 0], e[:, 1]
        big = np.abs(ad) >= FD_FLOOR * np.abs(ad).max()
        rel = np.abs(fd[big] - ad[big]) / np.abs(ad[big])
        absl = np.abs(fd[~big] - ad[~big]).max(initial=0.0) / np.abs(ad).max()
        print(f"adjoint vs FD ({name}): {big.sum()} of {len(e)} entries above the floor, per-entry rel max "
              f"{rel.max():.3e} median {np.median(rel):.3e}; below the floor max |fd-ad|/max|ad| {absl:.3e}")
        assert big.sum() >= len(e) // 3, name
        assert rel.max() < FD_RTOL, name
        # the absolute error of the central differences, measured 1.1e-7 (u*)
        # and 2.7e-7 (rho) of the largest gradient
        assert absl < 5e-7, name
    assert np.abs(np.concatenate([a.ravel() for a in u0])).max() > 0


def runtime_workloads():
    import __graft_entry__
    return __graft_entry__.load_package().workloads


def test_autograd_function_gradcheck(gpu_lib, capi, runtime, orc):
    """A torch.autograd.Function over the C-ABI forward and adjoint; inputs
    are the interior u*, v*, w* and rho of a periodic 16^3 box."""
    torch = pytest.importorskip("torch")
    n = 16
    d = capi.make_desc((n, n, n), rho1=1.0, rho2=1000.0)
    dt = 0.25 / n
    g = d.ng
    gpu = runtime.ParisGpu(d)

    def pad(x):
        a = np.zeros(orc.shape(d))
        a[g:g + n, g:g + n, g:g + n] = x
        orc.fill_ghosts(d, a)
        return a

    class Projection(torch.autograd.Function):
        @staticmethod
        def forward(ctx, us, vs, ws, rho):
            r = pad(rho.detach().numpy())
            ust = [pad(t.detach().numpy()) for t in (us, vs, ws)]
            gpu.upload(capi.F_RHO, r)
            out = gpu_forward(gpu, capi, dt, ust)
            ctx.rho, ctx.ust = r, ust
            return tuple(torch.from_numpy(np.ascontiguousarray(orc.interior(d, a))) for a in out)

        @staticmethod
        def backward(ctx, gu, gv, gw):
            gin = []
            for t in (gu, gv, gw):
                a = np.zeros(orc.shape(d))
                a[g:g + n, g:g + n, g:g + n] = t.numpy()
                gin.append(a)
            # the adjoint reads the forward state on the device (RHO, matrix,
            # P); other forwards may have run since, so restore it
            gpu.upload(capi.F_RHO, ctx.rho)
            gpu_forward(gpu, capi, dt, ctx.ust)
            gs, gb = gpu.projection_adjoint(dt, gin)
            grho = rho_chain(orc, d, ctx.rho, gb)
            return tuple(torch.from_numpy(np.ascontiguousarray(orc.interior(d, a))) for a in gs) + \
                (torch.from_numpy(grho),)

    rng = np.random.default_rng(4)
    us = [torch.tensor(rng.standard_normal((n, n, n)), requires_grad=True) for _ in range(3)]
    # a smooth density between 1 and 1000 plus 1% noise
    x = (np.arange(n) + 0.5) / n
    s3 = np.sin(2 * np.pi * x)[:, None, None] * np.sin(2 * np.pi * x)[None, :, None] * np.sin(2 * np.pi * x)
    r0 = (1.0 + 999.0 * (0.5 + 0.5 * s3)) * (1.0 + 0.01 * rng.standard_normal((n, n, n)))
    rho = torch.tensor(r0, requires_grad=True)
    try:
        assert torch.autograd.gradcheck(Projection.apply, (*us, rho), eps=1e-6, atol=1e-5, rtol=1e-4,
                                        fast_mode=True)
    finally:
        gpu.close()
