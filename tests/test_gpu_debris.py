"""clean_debris on the GPU against the oracle, bit for bit: methods 1 and 2
(a pass over the fractions as they were) and method 3 (in-place sweeps in the
reference's k, j, i order, run by wavefronts), on periodic and walled boxes.
(The reference's 2-D case, Nz = 2, is below the grid core's minimum of four
cells per direction.)"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def field(capi, orc, shape, bc, seed):
    d = capi.make_desc(shape, bc=bc)
    cvof, flag, _ = orc.init_spheres(d, [(0.4, 0.55, 0.5), (0.75, 0.3, 0.45)], [0.2, 0.1], refinement=4)
    rng = np.random.default_rng(seed)
    inner = orc.interior(d, cvof)
    # debris: a sprinkle of small fractions and of near-full cells
    m = rng.random(inner.shape)
    inner[m < 0.02] = rng.uniform(0.001, 0.2, inner.shape)[m < 0.02]
    inner[(m > 0.98)] = rng.uniform(0.8, 0.999, inner.shape)[m > 0.98]
    if bc == "periodic":
        orc.fill_ghosts(d, cvof)
    orc.flags_clip(d, cvof, flag)
    return d, cvof, flag


@pytest.mark.parametrize("shape,bc", [((24, 20, 16), "periodic"), ((24, 20, 16), "wall"), ((16, 24, 32), "wall")])
@pytest.mark.parametrize("method,nb", [(1, 2), (1, 1), (2, 2), (2, 1), (3, 2)])
def test_clean_debris_bitwise(gpu_lib, capi, runtime, orc, shape, bc, method, nb):
    d, cvof, flag = field(capi, orc, shape, bc, 11)
    ref_c, ref_f = cvof.copy(), flag.copy()
    sweeps_ref = orc.clean_debris(d, ref_c, ref_f, method, nb)
    with runtime.ParisGpu(d) as gpu:
        gpu.upload(capi.F_CVOF, cvof)
        gpu.upload(capi.F_VOF_FLAG, flag)
        sweeps = gpu.clean_debris(method, nb)
        out_c = gpu.download(capi.F_CVOF)
        out_f = gpu.download(capi.F_VOF_FLAG)
    assert sweeps == sweeps_ref
    assert np.array_equal(out_c, ref_c)
    if method == 3:
        assert np.array_equal(out_f, ref_f)
    assert (ref_c != cvof).any()   # the case cleans something
