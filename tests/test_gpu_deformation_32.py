"""The 32^3 deformation run on the device against the oracle, step by step.

Periodic unit cube, h = 1/32; a sphere of radius 0.15 at (0.35, 0.35, 0.35)
from ls2vof_refined with refinement 8 (vofmodules.f90:1195-1293); LeVeque's
three-dimensional deformation field with period 3 at the face centres, taken
at t + dt/2; dt = 0.25 h / 2, 768 steps to t = 3.  Every step, as the step
loop of the reference does it: rho = linfunc (arithmetic, 1 in the gas and
1000 in the liquid), SetupPoisson of the field, the reference multigrid
(NewSolverMG, MGsolver.f90:346-405) warm-started from the previous pressure,
project_velocity, then vofsweeps(itimestep) with the projected field
(vofmodules.f90:1340-1361; swpz / swpr, vofnonmodule.f90:126-237,664-754).

The field is solenoidal on the grid to rounding (its discrete divergence is
(2 - 1 - 1) sin(pi h)/h times a product of sines), so the right-hand side of
the pressure equation is rounding noise: it cannot be reduced relative to
itself, and the stopping test is absolute, 1e-10 of the divergence scale
RMS(u)/h.  One V-cycle meets it every step and the projection moves u by
rounding only.

The device and the oracle run free, each from its own previous step; the
test records per step max |dcvof| and the RMS of dcvof, the first step at
which max |dcvof| passes 1e-12, and the liquid volume sum(c) h^3 against
step 0 on both sides.  Measured on a B200: Weymouth-Yue stays within
2.5e-14 of the oracle for all 768 steps and holds the volume to 4.8e-14;
CIAM stays within 1e-12 until step 715 (6.3e-13 at the end) and its volume
grows by 4.08e-2, identically on both sides."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 32
STEPS = 768


def run(capi, runtime, orc, workloads, advect):
    n = N
    h = 1.0 / n
    dt = 0.25 * h / 2.0
    desc = capi.make_desc((n, n, n), rho1=1.0, rho2=1000.0, advect=advect)
    c_ref, f_ref, _ = orc.init_spheres(desc, [(0.35, 0.35, 0.35)], [0.15], refinement=8)
    p_ref = orc.zeros(desc)
    vol0 = orc.interior(desc, c_ref).sum() * h ** 3
    rows = []
    with runtime.ParisGpu(desc) as gpu:
        gpu.upload(capi.F_CVOF, c_ref)
        gpu.upload(capi.F_VOF_FLAG, f_ref)
        gpu.upload(capi.F_P, p_ref)
        for k in range(STEPS):
            u, v, w = workloads.deformation_faces((n, n, n), (k + 0.5) * dt)
            tol = 1e-10 * float(np.sqrt(np.mean(orc.interior(desc, u) ** 2))) / h
            # oracle
            rho = orc.linfunc(desc, c_ref, 1.0, 1000.0, capi.MEAN_ARITH)
            st, A = orc.setup_poisson(desc, u, v, w, rho, dt)
            assert st == 0
            st, it_ref, _, _ = orc.new_solver_mg(desc, A, p_ref, tol, maxit=50)
            assert st == 0
            uo, vo, wo = u.copy(), v.copy(), w.copy()
            orc.project_velocity(desc, uo, vo, wo, p_ref, rho, dt)
            orc.vofsweeps(desc, k + 1, dt, c_ref, f_ref, uo, vo, wo)
            # device
            for f, a in zip((capi.F_U, capi.F_V, capi.F_W), (u, v, w)):
                gpu.upload(f, a)
            gpu.linfunc(capi.F_RHO)
            gpu.setup_poisson(dt)
            r = gpu.new_solver(tol, maxit=50, mode=capi.MG_REFERENCE)
            gpu.project_velocity(dt)
            gpu.vof_sweeps(k + 1, dt)
            c = gpu.download(capi.F_CVOF)
            d = orc.interior(desc, c) - orc.interior(desc, c_ref)
            rows.append((k + 1, np.abs(d).max(), float(np.sqrt(np.mean(d * d))),
                         orc.interior(desc, c).sum() * h ** 3 / vol0 - 1.0,
                         orc.interior(desc, c_ref).sum() * h ** 3 / vol0 - 1.0, r.it, it_ref))
    return np.array(rows)


@pytest.mark.parametrize("advect,name", [(0, "CIAM"), (1, "Weymouth-Yue")])
def test_deformation_32_against_oracle(gpu_lib, capi, runtime, orc, workloads, advect, name):
    R = run(capi, runtime, orc, workloads, advect)
    step, dmax, drms, vgpu, vref, itg, itr = R.T
    over = np.nonzero(dmax > 1e-12)[0]
    first = int(step[over[0]]) if len(over) else None
    print(f"\n{name}: first step with max|dcvof| > 1e-12: {first}; largest max|dcvof| {dmax.max():.2e} "
          f"(step {int(step[np.argmax(dmax)])}); largest |volume drift| {np.abs(vgpu).max():.2e}")
    for s in (1, 10, 100, 200, 384, 500, 600, 700, 768):
        q = s - 1
        print(f"  step {s:4d}: max|dcvof| {dmax[q]:.2e}  rms {drms[q]:.2e}  volume drift device {vgpu[q]:+.3e} "
              f"oracle {vref[q]:+.3e}  V-cycles {int(itg[q])}/{int(itr[q])}")
    assert np.array_equal(itg, itr)
    if advect == 1:
        # Weymouth-Yue: within 1e-12 of the oracle over all 768 steps (2.5e-14
        # measured), the liquid volume held to 1e-13 on both sides (-4.8e-14)
        assert first is None
        assert np.abs(vgpu).max() <= 1e-13 and np.abs(vref).max() <= 1e-13
    else:
        # CIAM: within 1e-12 to step 714 (715 measured), 6.3e-13 at step 768;
        # the Lagrangian-explicit sweeps are not conservative under this
        # deformation: the volume grows by 4.08e-2 on both sides alike
        assert first is None or first >= 700
        assert dmax.max() <= 1e-11
        assert np.abs(vgpu - vref).max() <= 1e-11
        assert 0.03 < vgpu[-1] < 0.05
