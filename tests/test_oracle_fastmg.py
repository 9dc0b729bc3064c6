"""CPU tests of the oracle's restatement of the B200 multigrid (og_fastmg.c):
the smoother's relaxation factor on the levels below the finest."""
import numpy as np

from test_gpu_projection import drop_problem

N = 32
TOL = 1e-10


def _system(capi, orc, workloads):
    desc, cvof, rho, vel = drop_problem(capi, orc, workloads, N, bc="periodic", ndrops=4)
    _, A = orc.setup_poisson(desc, *vel, rho, 1e-3)
    return desc, A


def _solve(orc, desc, A, **kw):
    return orc.fastmg_solve(desc, A, np.zeros((N, N, N)), TOL, maxit=60, mixed=False, pcg=True, nu_coarse=4,
                            coarse_from=1, coarse_to=2, **kw)


def test_coarse_factor_equal_to_beta_is_the_same_cycle(capi, orc, workloads):
    """omega_coarse == omega is the cycle without it, bit for bit."""
    desc, A = _system(capi, orc, workloads)
    p0, it0, h0 = _solve(orc, desc, A, omega=1.1)
    p1, it1, h1 = _solve(orc, desc, A, omega=1.1, omega_coarse=1.1)
    assert it0 == it1 and np.array_equal(h0, h1) and np.array_equal(p0, p1)


def test_coarse_factor_changes_the_cycle_not_the_solution(capi, orc, workloads):
    """Another factor below the finest level gives another residual history,
    and the same pressure to the solver's tolerance."""
    desc, A = _system(capi, orc, workloads)
    p0, it0, h0 = _solve(orc, desc, A, omega=1.1)
    p1, it1, h1 = _solve(orc, desc, A, omega=1.1, omega_coarse=1.25)
    assert h1[-1] < TOL and h0[-1] < TOL
    assert not np.array_equal(h0[:min(it0, it1)], h1[:min(it0, it1)])
    d = (p1 - p1.mean()) - (p0 - p0.mean())
    assert np.abs(d).max() <= 1e-8 * np.abs(p0 - p0.mean()).max()
