"""Full-size parity fixture of the 3-D Laplacian workload from the oracle's complete solve.

Runs the oracle (the CPU restatement of EPSSolve with Krylov-Schur in
oracle/ks_oracle.c) on the 3-D 7-point Dirichlet Laplacian on a 128^3 grid
(n = 2,097,152), nev = 32 largest real, ncv = 80, tol = 1e-8, start vector
N(0,1) from seed 0 -- the benchmark workload -- and writes
laplacian3d_128_oracle.json with:
  * the converged eigenvalues and error estimates, restarts, Lanczos steps and
    Gram-Schmidt column visits of the solve;
  * each pair's residual ||Ax - lambda x|| / |lambda| computed in FP64 on the host;
  * for each eigenvector, its coefficients in the exact eigenspace of its
    eigenvalue (the orthonormal sine-product basis that
    slepc_b200.problems.laplacian_3d_eigenspace returns, in that order) and the
    norm of its component outside that eigenspace -- enough to compare another
    run's eigenvectors with these without storing 2M-long vectors;
  * the oracle's wall time, the thread count and the CPU it ran on.

Usage (from the repository root; about 7 minutes on 8 cores):
    python tests/golden/make_laplacian3d_fixture.py [threads]
"""
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from slepc_b200 import problems as P  # noqa: E402

N, NEV, NCV, TOL, SEED = 128, 32, 80, 1e-8, 0


def cpu_name():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def main(threads):
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    A = P.to_scipy(csr)
    v0 = P.start_vector(n, SEED)
    oracle.set_threads(threads)
    t0 = time.perf_counter()
    r = oracle.eps_solve(A, v0, nev=NEV, ncv=NCV, tol=TOL, which=oracle.LARGEST_REAL)
    wall = time.perf_counter() - t0
    pairs = []
    for i in range(r.nconv):
        lam, x = float(r.evals[i]), r.X[:, i]
        B = P.laplacian_3d_eigenspace(lam, N)
        coef = B.T @ x
        outside = float(np.linalg.norm(x - B @ coef))
        pairs.append({"eigenvalue": lam, "errest": float(r.errest[i]),
                      "residual": float(oracle.residual(A, x, lam)), "space_dim": int(B.shape[1]),
                      "coefficients": [float(c) for c in coef], "outside_norm": outside})
    out = {"workload": f"3-D 7-point Laplacian {N}^3, nev={NEV} largest real, ncv={NCV}, tol={TOL}, "
                       f"start vector N(0,1) seed {SEED}",
           "n": n, "nnz": int(csr[0][-1]), "nconv": r.nconv, "reason": r.reason, "its": r.its, "restarts": r.restarts,
           "lanczos_steps": r.lanczos_steps, "column_visits": r.column_visits,
           "wall_s": wall, "threads": threads, "cpu": cpu_name(), "pairs": pairs}
    path = os.path.join(HERE, "laplacian3d_128_oracle.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path}: nconv {r.nconv}, {r.its} restarts, {r.column_visits} column visits, {wall:.1f} s "
          f"on {threads} threads")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1))
