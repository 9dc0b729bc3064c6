"""Copies the golden vectors of the reference's own regression tests into
tests/golden/ (run once where the reference tree is available; the copies
are committed so that the tests need no reference tree).

  python make_fixtures.py <root of the slitvinov/paris-git tree>

  Tests/VOF/volumeref.txt        -> vof_volumeref.txt
  Tests/VOF/centerofmassref.txt  -> vof_centerofmassref.txt
  Tests/CylinderAdvection/reference.txt -> cylinder_advection_cvof.txt
      (cvof of the mid plane after 3800 steps, i outer and j inner, 16 x 16)
  Tests/CapWave/prosperetti      -> capwave_prosperetti.txt
      (Prosperetti's amplitude of the capillary wave against omega_0 t,
      the initial amplitude scaled to 0.01)
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    pairs = [("Tests/VOF/volumeref.txt", "vof_volumeref.txt"),
             ("Tests/VOF/centerofmassref.txt", "vof_centerofmassref.txt")]
    for src, dst in pairs:
        with open(os.path.join(ref_root, src)) as f:
            rows = [line.split() for line in f if line.strip()]
        with open(os.path.join(HERE, dst), "w") as f:
            f.write(f"# {src} of slitvinov/paris-git: time, value\n")
            for r in rows:
                f.write(f"{float(r[0]):.6e} {float(r[1]):.6e}\n")
        print("wrote", dst, len(rows), "rows")
    src, dst = "Tests/CylinderAdvection/reference.txt", "cylinder_advection_cvof.txt"
    with open(os.path.join(ref_root, src)) as f:
        vals = [line.strip() for line in f if line.strip()]
    with open(os.path.join(HERE, dst), "w") as f:
        f.write(f"# {src} of slitvinov/paris-git: cvof(i, j, (ks+ke)/2) at step 3800, i outer, j inner, "
                "as printed (E14.5)\n")
        for v in vals:
            f.write(v + "\n")
    print("wrote", dst, len(vals), "values")
    src, dst = "Tests/CapWave/prosperetti", "capwave_prosperetti.txt"
    with open(os.path.join(ref_root, src)) as f:
        rows = [line.split() for line in f if line.strip()]
    with open(os.path.join(HERE, dst), "w") as f:
        f.write(f"# {src} of slitvinov/paris-git: omega_0 t, amplitude (initial 0.01)\n")
        for r in rows:
            f.write(f"{r[0]} {r[1]}\n")
    print("wrote", dst, len(rows), "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_fixtures.py <root of the slitvinov/paris-git tree>")
    main(sys.argv[1])
