"""Build recipe of the CUDA library ``slepc_b200/libslepc_b200.so`` (sm_100a).

Compiles every source under ``slepc_b200/csrc`` with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and links the host LAPACK
(``dsteqr``/``dlartg``/``drot`` of the OpenBLAS that ships with scipy) used by
the projected-problem solver.  Objects go to ``slepc_b200/_build`` and the
shared library is written in place so it travels with the source tree.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libslepc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def openblas_path():
    import scipy

    libdir = os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError(f"scipy's bundled OpenBLAS not found under {libdir}")
    return cands[0]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


GEN_SRCS = [os.path.join(HERE, "gen_powerlaw.c"), os.path.join(HERE, "gen_knn.c")]
GEN_LIB = os.path.join(HERE, "libproblem_gen.so")


def build_generator(force=False):
    """Host-side generators of the test matrices (power-law rectangular, k-NN graph batches; gcc + OpenMP)."""
    if force or _stale(GEN_LIB, GEN_SRCS):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-Wall"] + GEN_SRCS +
                              ["-o", GEN_LIB, "-lm"])
    return GEN_LIB


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if verbose:
                cmd.append("-Xptxas=-v")
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        blas = openblas_path()
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
            "-Xlinker", "-rpath=" + os.path.dirname(blas), "--cudart=static", "-lpthread", "-ldl", "-lrt"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_generator(force="--force" in sys.argv))
