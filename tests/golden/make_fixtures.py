"""Copies the golden vectors of the reference's own regression tests into
tests/golden/ (run once where the reference tree is available; the copies
are committed so that the tests need no reference tree).

  Tests/VOF/volumeref.txt        -> vof_volumeref.txt
  Tests/VOF/centerofmassref.txt  -> vof_centerofmassref.txt
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
