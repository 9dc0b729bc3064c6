"""The on-disk formats written from the device fields, byte for byte against
the oracle's restatement of the Fortran formats (oracle/og_io.py): the
restart file of backup_VOF_write and the VTK files of output_VOF (both
DATASET kinds, plain and filtered).  backup_VOF_read into a fresh context
gives back the fields bit for bit (ES25.16E3 carries 17 significant digits);
a file of another grid is refused, as the reference stops on it."""
import numpy as np
import pytest

from oracle import og_io as io

pytestmark = pytest.mark.gpu


def state(capi, orc, bc):
    d = capi.make_desc((12, 10, 8), bc=bc, length=(1.2, 1.0, 0.8))
    cvof, flag, _ = orc.init_spheres(d, [(0.6, 0.5, 0.4)], [0.3], refinement=4)
    orc.flags_clip(d, cvof, flag)     # a state as a step leaves it: clipped, flags from cvof
    rng = np.random.default_rng(3)
    u, v, w, p = (rng.standard_normal(orc.shape(d)) for _ in range(4))
    orc.set_velocity_bc(d, u, v, w)
    return d, {"u": u, "v": v, "w": w, "p": p, "cvof": cvof, "flag": flag}


def upload(gpu, capi, st):
    for f in ("u", "v", "w", "p", "cvof"):
        gpu.upload(getattr(capi, "F_" + f.upper()), st[f])
    gpu.upload(capi.F_VOF_FLAG, st["flag"])


@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_backup_write_read(gpu_lib, capi, runtime, orc, tmp_path, bc):
    d, st = state(capi, orc, bc)
    fn = tmp_path / "backup_00000"
    fn.write_text("previous\n")
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, st)
        gpu.backup_vof_write(str(fn), 0.123456789, 42)
    assert (tmp_path / "backup_00000.old").read_text() == "previous\n"
    assert fn.read_text() == io.backup_text(d, st["u"], st["v"], st["w"], st["p"], st["cvof"], 0.123456789, 42)
    with runtime.ParisGpu(d) as gpu:
        t, it = gpu.backup_vof_read(str(fn))
        out = {f: gpu.download(getattr(capi, "F_" + f.upper())) for f in ("u", "v", "w", "p", "cvof")}
        flag = gpu.download(capi.F_VOF_FLAG)
    assert it == 42 and t == float(io.fortran_es(0.123456789, 17, 8, 3))
    g = d.ng
    inner = (slice(g, -g),) * 3
    for f in ("u", "v", "w", "p", "cvof"):
        assert np.array_equal(out[f][inner], st[f][inner]), f
    assert np.array_equal(out["p"], st["p"])                 # p is read with its ghosts
    assert np.array_equal(flag[inner], st["flag"][inner])
    # another grid is refused
    d2 = capi.make_desc((12, 10, 10), bc=bc)
    with runtime.ParisGpu(d2) as gpu:
        with pytest.raises(runtime.ParisError) as e:
            gpu.backup_vof_read(str(fn))
        assert e.value.status == capi.BAD_ARGS


@pytest.mark.parametrize("fmt", [2, 3])
@pytest.mark.parametrize("filtered", [False, True])
def test_vtk(gpu_lib, capi, runtime, orc, tmp_path, fmt, filtered):
    d, st = state(capi, orc, "wall")
    coords = orc.grid_coords(d)
    fn = tmp_path / "VOF00001-00000.vtk"
    with runtime.ParisGpu(d) as gpu:
        upload(gpu, capi, st)
        gpu.output_vof_vtk(str(fn), fmt, time=1.5, filtered=filtered)
        box = (3, 9, 2, 11, 4, 6)
        fn2 = tmp_path / "box.vtk"
        gpu.output_vof_vtk(str(fn2), fmt, time=0.0, index_range=box, filtered=filtered)
    assert fn.read_text() == io.vtk_text(d, st["cvof"], coords, fmt, 1.5, filtered=filtered)
    assert fn2.read_text() == io.vtk_text(d, st["cvof"], coords, fmt, 0.0, index_range=box, filtered=filtered)
