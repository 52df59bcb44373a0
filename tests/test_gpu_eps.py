"""End-to-end parity of the GPU Krylov-Schur solve with the CPU oracle.

Criteria (FP64 throughout):
  * every converged eigenvalue equals an oracle eigenvalue to 1e-10 relative
    (and, for Laplacians, an analytic eigenvalue to 1e-10);
  * for every cluster of equal eigenvalues, the GPU eigenspace and the oracle's
    eigenspace (the smaller one inside the larger one) agree: the sine of the
    largest principal angle is bounded by the Davis-Kahan bound of the two
    residuals over the gap to the rest of the spectrum, and below 1e-8 where
    that bound is;
  * every residual ||Ax - lambda x|| / |lambda| is <= tol, computed in FP64 on the
    host by the oracle and on the device by EPSComputeError.
Single-vector Krylov-Schur finds the copies of a multiple eigenvalue only
through rounding, so two correct runs can return different multiplicities;
the checks compare eigenspaces per cluster, not vectors per index.
"""
import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P
from tests import helpers as H

pytestmark = pytest.mark.gpu


def gpu_solve(csr, v0, nev, ncv, which, tol=1e-8, max_restarts=0):
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setDimensions(nev, ncv)
    E.setTolerances(tol)
    E.setWhichEigenpairs(which)
    E.setInitialSpace(v0)
    if max_restarts:
        E.setMaxRestarts(max_restarts)
    E.solve()
    nconv = E.getConverged()
    vals, vecs, errs = [], [], []
    for i in range(nconv):
        lam, x = E.getEigenpair(i)
        vals.append(lam)
        vecs.append(x)
        errs.append(E.computeError(i))
    X = np.stack(vecs, axis=1) if vecs else np.zeros((A.n, 0))
    out = dict(evals=np.array(vals), X=X, err=np.array(errs), nconv=nconv, its=E.getIterationNumber(),
               reason=E.getConvergedReason(), stats=E.getStats())
    E.destroy()
    A.destroy()
    return out


def check_parity(csr, g, o, oracle_mod, tol, analytic=None, gap_floor=None):
    As = P.to_scipy(csr)
    assert g["reason"] == S.CONVERGED_TOL and o.reason == oracle_mod.CONVERGED_TOL
    assert H.eig_set_match(g["evals"], o.evals, 0) < 1e-10
    assert H.eig_set_match(o.evals, g["evals"], 0) < 1e-10 or len(o.evals) != len(g["evals"])
    if analytic is not None:
        assert H.eig_set_match(g["evals"], analytic, 0) < 1e-10
    res = np.array([oracle_mod.residual(As, g["X"][:, i], g["evals"][i]) for i in range(g["nconv"])])
    assert res.max() <= tol, res.max()
    np.testing.assert_allclose(g["err"], res, rtol=1e-6, atol=1e-15)
    XtX = g["X"].T @ g["X"]
    assert np.abs(XtX - np.eye(g["nconv"])).max() < 1e-12
    # eigenspace agreement per cluster, against the Davis-Kahan bound
    spectrum = np.unique(np.round(analytic if analytic is not None else o.evals, 12))
    worst = 0.0
    for lam, s in H.eigenspace_sines(g["evals"], g["X"], o.evals, o.X, rtol=1e-9):
        others = spectrum[np.abs(spectrum - lam) > 1e-9 * abs(lam)]
        gap = np.abs(others - lam).min() if len(others) else abs(lam)
        bound = 2 * tol * abs(lam) / gap
        assert s <= max(bound, 1e-8), (lam, s, bound)
        worst = max(worst, s)
    return worst


def test_ex2_golden_gpu(oracle_mod):
    """ex2.c -n 72 -eps_nev 4 -eps_ncv 20 on the GPU prints SLEPc's golden digits."""
    gold = H.golden("ex2_1.json")
    csr = P.laplacian_2d(72)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 0)
    g = gpu_solve(csr, v0, 4, 20, S.LARGEST_MAGNITUDE)
    got = [float("%.5f" % v) for v in g["evals"][:4]]
    assert got in [o["values"] for o in gold["outputs"].values()]
    o = oracle_mod.eps_solve(P.to_scipy(csr), v0, nev=4, ncv=20, which=oracle_mod.LARGEST_MAGNITUDE)
    check_parity(csr, g, o, oracle_mod, 1e-8, analytic=P.laplacian_2d_eigs(72))
    assert abs(g["its"] - o.its) <= 2


def test_config1_2d_laplacian_100(oracle_mod):
    """2-D 5-point Laplacian 100x100, nev=10 largest magnitude, ncv=32, tol=1e-8."""
    csr = P.laplacian_2d(100)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 0)
    g = gpu_solve(csr, v0, 10, 32, S.LARGEST_MAGNITUDE)
    o = oracle_mod.eps_solve(P.to_scipy(csr), v0, nev=10, ncv=32, which=oracle_mod.LARGEST_MAGNITUDE)
    assert g["nconv"] >= 10
    check_parity(csr, g, o, oracle_mod, 1e-8, analytic=P.laplacian_2d_eigs(100))


@pytest.mark.parametrize("N,seed", [(16, 0), (24, 1)])
def test_3d_laplacian_nev32_ncv80(oracle_mod, N, seed):
    """The 3-D 7-point Laplacian workload (nev=32 largest real, ncv=80) on small grids."""
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, seed)
    g = gpu_solve(csr, v0, 32, 80, S.LARGEST_REAL)
    o = oracle_mod.eps_solve(P.to_scipy(csr), v0, nev=32, ncv=80, which=oracle_mod.LARGEST_REAL)
    assert g["nconv"] >= 32
    check_parity(csr, g, o, oracle_mod, 1e-8, analytic=P.laplacian_3d_eigs(N))


def test_random_sparse_vs_dense_eigh(oracle_mod):
    """Random symmetric sparse matrix: GPU eigenvalues equal dense LAPACK to 1e-10 (pins beyond the oracle)."""
    import scipy.sparse as sp

    rng = np.random.default_rng(11)
    n = 1200
    B = sp.random(n, n, density=0.01, random_state=rng, format="csr")
    A = (B + B.T + sp.diags(rng.standard_normal(n))).tocsr()
    A.sort_indices()
    csr = (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data)
    v0 = P.start_vector(n, 3)
    for which, key in ((S.LARGEST_MAGNITUDE, lambda e: -np.abs(e)), (S.SMALLEST_REAL, lambda e: e),
                       (S.LARGEST_REAL, lambda e: -e)):
        g = gpu_solve(csr, v0, 6, 30, which)
        ev = np.linalg.eigvalsh(A.toarray())
        top = ev[np.argsort(key(ev), kind="stable")][:6]
        np.testing.assert_allclose(g["evals"][:6], top, rtol=1e-10)
        o = oracle_mod.eps_solve(A, v0, nev=6, ncv=30, which=which)
        check_parity(csr, g, o, oracle_mod, 1e-8, analytic=ev)


def test_solve_csr_host_entry_point(oracle_mod):
    """The one-call host-buffer entry point returns the same pairs as the object API."""
    csr = P.laplacian_2d(50)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 5)
    r = S.solve_csr_host(csr, v0, 6, 24, which=S.LARGEST_MAGNITUDE)
    g = gpu_solve(csr, v0, 6, 24, S.LARGEST_MAGNITUDE)
    assert r["nconv"] == g["nconv"] and r["its"] == g["its"]
    np.testing.assert_allclose(r["evals"], g["evals"], rtol=1e-13)


def test_max_iterations_and_restart_cap():
    csr = P.laplacian_2d(60)
    n = len(csr[0]) - 1
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(12, 30)
    E.setTolerances(1e-14, 3)
    E.setInitialSpace(P.start_vector(n, 0))
    E.solve()
    assert E.getConvergedReason() == S.DIVERGED_ITS and E.getIterationNumber() == 3


def test_zero_initial_vector_is_an_error():
    csr = P.laplacian_2d(20)
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(2, 10)
    E.setInitialSpace(np.zeros(A.n))
    with pytest.raises(S.B200Error) as ei:
        E.solve()
    assert ei.value.status == 5


def test_invariant_subspace_breakdown_restarts():
    """A start vector inside a 3-dimensional invariant subspace: Lanczos breaks down after 3 steps,
    the solver restarts from a random vector (EPSGetStartVector, epssolve.c:841) and still converges."""
    n = 400
    d = np.arange(1.0, n + 1.0)
    csr = (np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d)
    v0 = np.zeros(n)
    v0[[n - 1, n - 2, n - 3]] = 1.0
    g = gpu_solve(csr, v0, 5, 20, S.LARGEST_MAGNITUDE)
    assert g["reason"] == S.CONVERGED_TOL
    np.testing.assert_allclose(np.sort(g["evals"][:5])[::-1], d[::-1][:5], rtol=1e-10)


@pytest.mark.parametrize("N", [128])
def test_config2_full_size_properties(N):
    """3-D 128^3 Laplacian (n=2,097,152), nev=32 largest real, ncv=80: size-independent properties --
    eigenvalues on the analytic spectrum to 1e-10, residuals <= 1e-8 (device EPSComputeError, FP64),
    orthonormal eigenvectors."""
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    g = gpu_solve(csr, P.start_vector(n, 0), 32, 80, S.LARGEST_REAL)
    assert g["reason"] == S.CONVERGED_TOL and g["nconv"] >= 32
    assert H.eig_set_match(g["evals"], P.laplacian_3d_eigs(N), 0) < 1e-10
    assert g["err"].max() <= 1e-8
    XtX = g["X"].T @ g["X"]
    assert np.abs(XtX - np.eye(g["nconv"])).max() < 1e-12
