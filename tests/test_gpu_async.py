"""Asynchronous transfers: an uploaded field takes its values at the commit,
for the work issued after it; a download snapshots the field as the work
issued before it left it; a pipeline of uploads (started a step early),
commits, steps and downloads gives the same fields as the synchronous calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ordering_against_the_handle_stream(gpu_lib, capi, runtime, orc):
    d = capi.make_desc((32, 24, 16))
    rng = np.random.default_rng(1)
    a, b = (np.ascontiguousarray(rng.standard_normal(orc.shape(d))) for _ in range(2))
    snap1, snap1b, snap2, snap3 = (np.empty(orc.shape(d)) for _ in range(4))
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_U, a)
        gpu.download_async(capi.F_U, snap1)     # a
        gpu.upload_async(capi.F_U, b)
        gpu.download_async(capi.F_U, snap2)     # still a: not committed yet
        gpu.upload_commit(capi.F_U)             # u = b for what follows
        gpu.download_async(capi.F_U, snap1b)    # b
        gpu.copy_field(capi.F_V, capi.F_U)      # v = b
        gpu.fill_field(capi.F_U, 3.0)
        gpu.download_async(capi.F_V, snap3)     # b
        gpu.upload_async(capi.F_W, a)
        gpu.upload_commit(capi.F_W)
        gpu.sync_transfers()
        w = gpu.download(capi.F_W)
        u = gpu.download(capi.F_U)
    assert np.array_equal(snap1, a) and np.array_equal(snap2, a)
    assert np.array_equal(snap1b, b) and np.array_equal(snap3, b)
    assert np.array_equal(w, a) and np.all(u == 3.0)


def test_pipelined_steps_match_the_synchronous_calls(gpu_lib, capi, runtime, orc, workloads):
    n, steps = 32, 4
    d = capi.make_desc((n, n, n), rho1=1.0, rho2=1000.0)
    cen, rad = workloads.drop_layout(4, rmin=0.1, rmax=0.2, seed=0, h=1.0 / n)
    rng = np.random.default_rng(2)
    us = [np.ascontiguousarray(orc.zeros(d) + rng.standard_normal(orc.shape(d))) for _ in range(3)]
    for a in us:
        orc.fill_ghosts(d, a)
    dt = 1e-3

    def step(gpu, k):
        for dst, src in ((capi.F_U, capi.F_USTAR), (capi.F_V, capi.F_VSTAR), (capi.F_W, capi.F_WSTAR)):
            gpu.copy_field(dst, src)
        gpu.vof_sweeps(k, dt)
        gpu.linfunc(capi.F_RHO)
        gpu.setup_poisson(dt)
        gpu.fill_field(capi.F_P, 0.0)
        gpu.new_solver(0.0, maxit=100, mode=capi.MG_MIXED, rel_tol=1e-10, pcg=1)
        gpu.project_velocity(dt)

    outs = (capi.F_U, capi.F_V, capi.F_W, capi.F_CVOF)
    ref = []
    with runtime.ParisGpu(d) as gpu:
        gpu.init_spheres(cen, rad, refinement=4)
        for k in range(steps):
            for f, a in zip((capi.F_USTAR, capi.F_VSTAR, capi.F_WSTAR), us):
                gpu.upload(f, a * (1.0 + 0.1 * k))
            step(gpu, k)
            ref.append([gpu.download(f) for f in outs])
    ins = [[np.ascontiguousarray(a * (1.0 + 0.1 * k)) for a in us] for k in range(steps)]
    got = [[np.empty(orc.shape(d)) for _ in outs] for _ in range(steps)]
    with runtime.ParisGpu(d) as gpu:
        gpu.init_spheres(cen, rad, refinement=4)
        stars = (capi.F_USTAR, capi.F_VSTAR, capi.F_WSTAR)
        for f, a in zip(stars, ins[0]):
            gpu.upload_async(f, a)
        for k in range(steps):
            for f in stars:
                gpu.upload_commit(f)
            if k + 1 < steps:           # the next step's inputs go up during this step
                for f, a in zip(stars, ins[k + 1]):
                    gpu.upload_async(f, a)
            step(gpu, k)
            for f, h in zip(outs, got[k]):
                gpu.download_async(f, h)
        gpu.sync_transfers()
    for k in range(steps):
        for a, b in zip(got[k], ref[k]):
            assert np.array_equal(a, b), k
