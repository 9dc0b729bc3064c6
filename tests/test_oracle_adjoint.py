"""The oracle's projection adjoint against central finite differences of its
own forward projection in the face-coefficient form (no GPU needed): the
CPU reference gradient the GPU adjoint is compared with."""
import numpy as np
import pytest

FD_RTOL = 1e-6


@pytest.mark.parametrize("bc", ["periodic", "wall"])
def test_oracle_adjoint_vs_fd(capi, orc, bc):
    n = 16
    d = capi.make_desc((n, n, n), bc=bc)
    rng = np.random.default_rng(0)
    cvof, _, _ = orc.init_spheres(d, [(0.4, 0.45, 0.5), (0.7, 0.3, 0.6)], [0.2, 0.15], refinement=4)
    rho = orc.linfunc(d, cvof, 1.0, 1000.0, capi.MEAN_ARITH)
    orc.fill_ghosts(d, rho)
    m = [orc.updated_faces(d, k) for k in range(3)]
    us = [rng.standard_normal(orc.shape(d)) for _ in range(3)]
    w = [rng.standard_normal(orc.shape(d)) for _ in range(3)]
    for a, b, mk in zip(us, w, m):
        a[~mk] = 0.0    # wall faces carry u = 0; ghosts are not parameters
        b[~mk] = 0.0
    dt = 1e-3
    B = orc.face_B(d, rho)
    _, p, it = orc.projection_forward_B(d, dt, B, us)
    assert it < 60
    gs, gb, _ = orc.projection_adjoint(d, dt, B, p, w)
    for a, b, mk in zip(gs + gb, gs + gb, m + m):
        assert np.all(a[~mk] == 0.0)

    def fd(kind, k, q):
        eps = 1e-6 if kind == "u" else 1e-6 * B[k][q]
        out = []
        for s in (1.0, -1.0):
            uu = [a.copy() for a in us]
            bb = [a.copy() for a in B]
            (uu if kind == "u" else bb)[k][q] += s * eps
            out.append(orc.projection_forward_B(d, dt, bb, uu)[0])
        return sum(float((a * (b - c))[mk].sum()) for a, b, c, mk in zip(w, out[0], out[1], m)) / (2 * eps)

    for kind, grad in (("u", gs), ("B", gb)):
        pairs = []
        for _ in range(25):
            k = int(rng.integers(3))
            idx = np.argwhere(m[k])
            q = tuple(idx[rng.integers(len(idx))])
            pairs.append((fd(kind, k, q), grad[k][q]))
        e = np.array(pairs)
        rel = np.abs(e[:, 0] - e[:, 1]).max() / np.abs(e[:, 1]).max()
        assert rel < FD_RTOL, (kind, rel)


def test_oracle_adjoint_is_a_transpose(capi, orc):
    """<g, J du*> = <J^T g, du*> for the linear map u* -> u at fixed B."""
    n = 8
    d = capi.make_desc((n, n, n))
    rng = np.random.default_rng(1)
    rho = orc.zeros(d) + 1.0 + 999.0 * rng.uniform(size=orc.shape(d))
    orc.fill_ghosts(d, rho)
    B = orc.face_B(d, rho)
    m = [orc.updated_faces(d, k) for k in range(3)]
    du = [np.where(mk, rng.standard_normal(orc.shape(d)), 0.0) for mk in m]
    g = [np.where(mk, rng.standard_normal(orc.shape(d)), 0.0) for mk in m]
    dt = 0.01
    Jdu, p, _ = orc.projection_forward_B(d, dt, B, du)
    gs, _, _ = orc.projection_adjoint(d, dt, B, p, g)
    lhs = sum(float((a * b)[mk].sum()) for a, b, mk in zip(g, Jdu, m))
    rhs = sum(float((a * b)[mk].sum()) for a, b, mk in zip(gs, du, m))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1.0)
