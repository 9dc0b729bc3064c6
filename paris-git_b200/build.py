"""Compiles libparis_b200.so in-tree with nvcc for sm_100a.

Translation units that must reproduce the reference's floating-point results
bit for bit are compiled with -fmad=false; the B200 multigrid keeps FMA.
"""
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libparis_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]
# sources and whether they keep the reference's operation order (no FMA)
SOURCES = {
    "ctx.cu": True,
    "poisson.cu": True,
    "mg_ref.cu": True,
    "mg_fast.cu": False,
    "solver.cu": True,
    "vof.cu": True,
    "adjoint.cu": True,
    "noalloc.cu": True,
    "st.cu": True,
    "momentum.cu": True,
    "stats.cu": True,
    "io.cu": True,
    "debris.cu": True,
    "momcons.cu": True,
}


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _compile(src, exact, verbose=False):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *COMMON, "-c", os.path.join(CSRC, src), "-o", obj]
    if exact:
        cmd.insert(1, "-fmad=false")
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    return obj, r.stderr


def build_library(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        results = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), SOURCES.items()))
    objs = [o for o, _ in results]
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    if verbose:
        for (src, _), (_, log) in zip(SOURCES.items(), results):
            print(f"== {src}\n{log}")
    return LIB


if __name__ == "__main__":
    import sys
    print(build_library(verbose="-v" in sys.argv))
