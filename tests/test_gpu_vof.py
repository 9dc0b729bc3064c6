"""Parity of the VOF kernels on the GPU against the FP64 oracle.

The split sweeps (CIAM and Weymouth-Yue), the flags, the boundary ghosts and
the sphere initialisation must agree with the oracle to 1e-12 in cvof (the
transcendental functions of AL3D may differ by an ulp between the device and
glibc) and exactly in the flags.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def setup(capi, orc, workloads, n=24, bc="periodic", advect=0, vofbc=None, seed=0):
    desc = capi.make_desc((n, n, n), bc=bc, vofbc=vofbc, advect=advect)
    cen, rad = workloads.drop_layout(5, rmin=0.1, rmax=0.18, seed=seed, h=1.0 / n)
    cvof, flag, _ = orc.init_spheres(desc, cen, rad, refinement=4)
    return desc, cvof, flag, cen, rad


def velocity(capi, orc, workloads, desc, t=0.3):
    u, v, w = workloads.deformation_faces((desc.nx, desc.ny, desc.nz), t)
    return u, v, w


@pytest.mark.parametrize("advect", [0, 1])
@pytest.mark.parametrize("tswap", [0, 1, 2])
def test_sweeps_periodic(gpu_lib, capi, runtime, orc, workloads, advect, tswap):
    desc, cvof, flag, _, _ = setup(capi, orc, workloads, advect=advect)
    u, v, w = velocity(capi, orc, workloads, desc)
    dt = 0.25 / desc.nx / 2.0
    ref_c, ref_f = cvof.copy(), flag.copy()
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        for f, a in zip((capi.F_U, capi.F_V, capi.F_W), (u, v, w)):
            gpu.upload(f, a)
        for step in range(3):
            orc.vofsweeps(desc, tswap + step, dt, ref_c, ref_f, u, v, w)
            gpu.vof_sweeps(tswap + step, dt)
        c = gpu.download(capi.F_CVOF)
        f = gpu.download(capi.F_VOF_FLAG)
    assert np.abs(c - ref_c).max() <= TOL
    assert np.array_equal(f, ref_f)


@pytest.mark.parametrize("vofbc", [(0, 0, 0, 0, 0, 0), (1, 0, 4, 4, 1, 0)])
def test_sweeps_walls(gpu_lib, capi, runtime, orc, workloads, vofbc):
    desc, cvof, flag, _, _ = setup(capi, orc, workloads, bc="wall", vofbc=vofbc)
    u, v, w = velocity(capi, orc, workloads, desc)
    dt = 0.25 / desc.nx / 2.0
    ref_c, ref_f = cvof.copy(), flag.copy()
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        for f, a in zip((capi.F_U, capi.F_V, capi.F_W), (u, v, w)):
            gpu.upload(f, a)
        for step in range(3):
            orc.vofsweeps(desc, step, dt, ref_c, ref_f, u, v, w)
            gpu.vof_sweeps(step, dt)
        c = gpu.download(capi.F_CVOF)
        f = gpu.download(capi.F_VOF_FLAG)
    assert np.abs(c - ref_c).max() <= TOL
    assert np.array_equal(f, ref_f)


@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_init_spheres(gpu_lib, capi, runtime, orc, workloads, bc):
    desc, _, _, cen, rad = setup(capi, orc, workloads, n=32, bc=bc)
    c_ref, f_ref, _ = orc.init_spheres(desc, cen, rad, refinement=8, jacobi=True)
    with runtime.ParisGpu(desc) as gpu:
        gpu.init_spheres(cen, rad, refinement=8)
        c = gpu.download(capi.F_CVOF)
        f = gpu.download(capi.F_VOF_FLAG)
    assert np.abs(c - c_ref).max() <= TOL
    assert np.array_equal(f, f_ref)


JET, DEG90, DRY, OUT = 2, 5, 0, 4


@pytest.mark.parametrize("advect", [0, 1])
@pytest.mark.parametrize("vofbc", [(JET, DEG90, DRY, DEG90, OUT, DEG90), (DEG90, DEG90, DEG90, DEG90, DEG90, DEG90)])
def test_sweeps_jet_and_90deg(gpu_lib, capi, runtime, orc, workloads, advect, vofbc):
    """'jet' and '90deg' faces (vofmodules.f90:1716-1720,1758-1811): the first
    ghost layer from the inflow pattern or the adjacent cell, the second kept
    from before the sweep.  The state starts from drops in a dry box whose
    second ghost layers are set to distinct values, with an inflow through
    x- so that the jet's first layer is advected in."""
    n = 24
    jet = (2, 0.5, 0.45, 0.2, 0.0)
    dry = capi.make_desc((n, n, n), bc="wall", advect=advect)
    desc = capi.make_desc((n, n, n), bc="wall", vofbc=vofbc, advect=advect, jet=jet)
    cen, rad = workloads.drop_layout(5, rmin=0.1, rmax=0.18, seed=3, h=1.0 / n, margin_cells=0)
    cvof, flag, _ = orc.init_spheres(dry, cen, rad, refinement=4)
    rng = np.random.default_rng(7)
    for sl in ((slice(None), slice(None), 0), (slice(None), slice(None), -1), (slice(None), 0, slice(None)),
               (slice(None), -1, slice(None)), (0, slice(None), slice(None)), (-1, slice(None), slice(None))):
        cvof[sl] = rng.choice([0.0, 1.0, 0.4], size=cvof[sl].shape)
    orc.setvofbc(desc, cvof, flag)
    orc.flags_clip(desc, cvof, flag)
    u, v, w = velocity(capi, orc, workloads, desc)
    u = u + 0.6
    dt = 0.25 / n / 2.0
    ref_c, ref_f = cvof.copy(), flag.copy()
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        for f, a in zip((capi.F_U, capi.F_V, capi.F_W), (u, v, w)):
            gpu.upload(f, a)
        for step in range(3):
            orc.vofsweeps(desc, step, dt, ref_c, ref_f, u, v, w)
            gpu.vof_sweeps(step, dt)
        c = gpu.download(capi.F_CVOF)
        f = gpu.download(capi.F_VOF_FLAG)
    assert np.abs(c - ref_c).max() <= TOL
    assert np.array_equal(f, ref_f)
    if vofbc[0] == JET:   # the jet carried liquid into the first interior column
        assert ref_c[2:-2, 2:-2, 2].sum() > cvof[2:-2, 2:-2, 2].sum()


@pytest.mark.parametrize("code", [JET, DEG90])
def test_init_spheres_refuses_jet_and_90deg(gpu_lib, capi, runtime, code):
    desc = capi.make_desc((16, 16, 16), bc="wall", vofbc=(code, 0, 0, 0, 0, 0), jet=(2, 0.5, 0.5, 0.2, 0.0))
    with runtime.ParisGpu(desc) as gpu:
        with pytest.raises(runtime.ParisError, match="bad flag"):
            gpu.init_spheres([(0.5, 0.5, 0.5)], [0.25], refinement=8)
