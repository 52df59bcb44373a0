"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/ks_oracle.c`` with gcc + OpenMP into ``oracle/liboracle.so``,
linked against the OpenBLAS that ships inside scipy (LAPACK ``dsteqr``,
``dlartg``, ``drot``, ``dsytrd``, ``dorgtr`` and BLAS ``dgemv``/``dgemm``
exported with a ``scipy_`` prefix).

SLEPc's own sources cannot be compiled here: they need PETSc headers and
libraries, which the image does not contain, so there is no ``oracle/_ref``
build of the reference itself.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "ks_oracle.c")


def openblas_path():
    import scipy

    libdir = os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError(f"scipy's bundled OpenBLAS not found under {libdir}")
    return cands[0]


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    blas = openblas_path()
    cmd = [
        "gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-Wall",
        SRC, "-o", LIB,
        "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
        "-Wl,-rpath," + os.path.dirname(blas), "-lm",
    ]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
