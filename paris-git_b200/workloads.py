"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference has no such generators; these build the fields the harness
feeds through the C-ABI.  Host arrays are in the reference layout
(Nzt, Nyt, Nxt) float64 with Ng=2 ghost layers, i fastest.
"""
import numpy as np


def ghosted_shape(n, ng=2):
    return (n[2] + 2 * ng, n[1] + 2 * ng, n[0] + 2 * ng)


def fill_periodic_ghosts(a, ng=2, periodic=(True, True, True)):
    """do_all_ghost on one rank for periodic directions (x, then y, then z)."""
    # x is the last numpy axis
    for ax, per in ((2, periodic[0]), (1, periodic[1]), (0, periodic[2])):
        if not per:
            continue
        n = a.shape[ax] - 2 * ng
        sl = [slice(None)] * 3
        src = [slice(None)] * 3
        sl[ax] = slice(0, ng)
        src[ax] = slice(n, n + ng)
        a[tuple(sl)] = a[tuple(src)]
        sl[ax] = slice(n + ng, n + 2 * ng)
        src[ax] = slice(ng, 2 * ng)
        a[tuple(sl)] = a[tuple(src)]
    return a


def drop_layout(ndrops=64, rmin=0.03, rmax=0.08, seed=0, h=1.0 / 256, box=(1.0, 1.0, 1.0),
                margin_cells=2):
    """Seeded non-overlapping drops: radii U[rmin,rmax], centres U in the box by
    rejection, pairwise distance > r_i + r_j + 2h, each drop at least
    margin_cells cells inside the box (the level set of the reference,
    shapes2ls, is not periodic)."""
    rng = np.random.default_rng(seed)
    centers, radii = [], []
    tries = 0
    while len(radii) < ndrops:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place drops")
        r = rng.uniform(rmin, rmax)
        lo = r + margin_cells * h
        c = np.array([rng.uniform(lo, L - lo) for L in box])
        ok = True
        for c2, r2 in zip(centers, radii):
            if np.linalg.norm(c - c2) <= r + r2 + 2 * h:
                ok = False
                break
        if ok:
            centers.append(c)
            radii.append(r)
    return np.array(centers), np.array(radii)


def smoothed_gaussian_faces(n, seed=1, sweeps=3, ng=2):
    """u*, v*, w*: i.i.d. N(0,1) per face, then `sweeps` Jacobi sweeps
    u <- (u + sum of the 6 face neighbours)/7 on the periodic grid.
    Returns three ghosted arrays with periodic ghosts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(3):
        u = rng.standard_normal((n[2], n[1], n[0]))
        for _ in range(sweeps):
            u = (u + np.roll(u, 1, 0) + np.roll(u, -1, 0) + np.roll(u, 1, 1) + np.roll(u, -1, 1)
                 + np.roll(u, 1, 2) + np.roll(u, -1, 2)) / 7.0
        a = np.zeros(ghosted_shape(n, ng))
        a[ng:ng + n[2], ng:ng + n[1], ng:ng + n[0]] = u
        fill_periodic_ghosts(a, ng)
        out.append(a)
    return out


def deformation_faces(n, t, period=3.0, ng=2, length=1.0):
    """The 3-D deformation field of LeVeque at time t, evaluated at the face
    centres of the staggered grid (u at (xh(i), y(j), z(k)) etc.):
      u =  2 sin^2(pi x) sin(2 pi y) sin(2 pi z) cos(pi t / T)
      v = -sin(2 pi x) sin^2(pi y) sin(2 pi z) cos(pi t / T)
      w = -sin(2 pi x) sin(2 pi y) sin^2(pi z) cos(pi t / T)"""
    h = length / n[0]
    idx = np.arange(-ng, n[0] + ng)
    xc = (idx + 0.5) * h      # cell centres
    xf = (idx + 1.0) * h      # face i+1/2
    ct = np.cos(np.pi * t / period)
    pi = np.pi
    Z, Y, X = np.meshgrid(xc, xc, xf, indexing="ij")
    u = 2 * np.sin(pi * X) ** 2 * np.sin(2 * pi * Y) * np.sin(2 * pi * Z) * ct
    Z, Y, X = np.meshgrid(xc, xf, xc, indexing="ij")
    v = -np.sin(2 * pi * X) * np.sin(pi * Y) ** 2 * np.sin(2 * pi * Z) * ct
    Z, Y, X = np.meshgrid(xf, xc, xc, indexing="ij")
    w = -np.sin(2 * pi * X) * np.sin(2 * pi * Y) * np.sin(pi * Z) ** 2 * ct
    return [np.ascontiguousarray(a) for a in (u, v, w)]
