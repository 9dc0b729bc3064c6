"""The reference's Tests/CapWave case (inputshort): a cosine interface of
amplitude one cell at y = 1.5 in a 1 x 3 x 0.0625 box of 32 x 96 x 2 cubic cells, equal
densities and viscosities (rho 1, mu 0.0182571749236), sigma 1, periodic
velocity, dry/wet VOF ghosts in y and z, dt = 0.0003042906 up to
t = 0.560655281 (1843 steps), the interface height sampled every 10 steps as
interface_max_min does (paris.f90:1076-1111).  The amplitude, scaled to 0.01
at t = 0, is compared with Prosperetti's solution of the initial-value
problem (tests/golden/capwave_prosperetti.txt, the reference's own data),
sample by sample (the samples are omega_0 * 10 dt apart, as its rows are)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DT = 0.0003042906
END = 0.560655281
NX, NY, NZ = 32, 96, 2


def desc(capi):
    vb = [capi.VOFBC_PERIODIC, capi.VOFBC_WET, capi.VOFBC_WET, capi.VOFBC_PERIODIC, capi.VOFBC_DRY,
          capi.VOFBC_DRY]
    return capi.make_desc((NX, NY, NZ), length=(1.0, 3.0, 0.0625), bc="periodic", vofbc=vb, rho1=1.0,
                          rho2=1.0, mu1=0.0182571749236, mu2=0.0182571749236, sigma=1.0)


def theory():
    with open(os.path.join(HERE, "golden", "capwave_prosperetti.txt")) as f:
        return np.array([[float(v) for v in line.split()] for line in f if line.strip() and not line.startswith("#")])


def interface_max_y(d, cvof):
    """interface_max_min: the largest y(j) + dy (c(j) - 0.5) over the cells
    (i, j, k) of j = js..je-10 whose fraction differs from that of j+1."""
    g = d.ng
    h = 3.0 / NY
    best = -1e7
    for j in range(g, g + NY - 10):
        a, b = cvof[g:-g, j, g:-g], cvof[g:-g, j + 1, g:-g]
        m = np.abs(a - b) > 1e-10
        if m.any():
            yj = (j - g + 0.5) * h
            best = max(best, float((yj + h * (a[m] - 0.5)).max()))
    return best


def run(step, read_cvof):
    """Steps until t >= END; returns the scaled amplitudes of the samples."""
    samples = [interface_max_y(*read_cvof())]
    t, k = 0.0, 0
    while t < END:
        k += 1
        t += DT
        step(k)
        if k % 10 == 0 and t < END:
            samples.append(interface_max_y(*read_cvof()))
    s = np.array(samples)
    return (s - 1.5) / (s[0] - 1.5) * 0.01


def rms_against_theory(amp):
    th = theory()[: len(amp), 1]
    return float(np.sqrt(np.mean((amp - th) ** 2)))
