"""Mixed-precision Krylov-Schur (EPS.Precision.MIXED) against FP64 references.

The mixed form runs its Krylov-Schur phase on an FP32 basis with FP32 matrix
values and then refines the block of leading Ritz vectors in FP64, so its
results are compared with FP64 references by property, not bit for bit:
  * every residual ||Ax - lambda x|| / |lambda| computed in FP64 on the host
    (the oracle's residual) is <= tol, and the device's EPSComputeError agrees;
  * every eigenvalue lies on the exact spectrum (analytic for the Laplacians,
    dense LAPACK otherwise) to 1e-10 relative;
  * the distinct values found are the leading distinct values of the exact
    spectrum to 1e-10 (none skipped); whether every copy of a repeated
    eigenvalue was found is reported (the block refinement often recovers
    copies a single-vector Krylov run misses, but not always);
  * the eigenvectors are orthonormal to 1e-12 and each lies in its exact
    eigenspace within the Davis-Kahan bound (residual / gap, floor 1e-8);
  * the error of each eigenvalue against the FP64 oracle's run is reported.
"""
import json
import os

import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P
from tests import helpers as H

pytestmark = pytest.mark.gpu


def mixed_solve(csr, v0, nev, ncv, which, tol=1e-8, dtype=None, **opts):
    n = len(csr[0]) - 1
    A = S.Mat().createAIJ(csr, size=(n, n), dtype=dtype) if dtype is not None else S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setDimensions(nev, ncv)
    E.setTolerances(tol)
    E.setWhichEigenpairs(which)
    E.setInitialSpace(v0)
    E.setPrecision(S.EPS.Precision.MIXED)
    if opts:
        E.setMixedOptions(**opts)
    E.solve()
    nconv = E.getConverged()
    vals, vecs, errs = [], [], []
    for i in range(nconv):
        lam, x = E.getEigenpair(i)
        vals.append(lam)
        vecs.append(x)
        errs.append(E.computeError(i))
    out = dict(evals=np.array(vals), X=np.stack(vecs, axis=1) if vecs else np.zeros((n, 0)), err=np.array(errs),
               nconv=nconv, reason=E.getConvergedReason(), stats=E.getStats())
    E.destroy()
    A.destroy()
    return out


def _report(name, **kv):
    path = os.environ.get("PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"test": name, **kv}) + "\n")


def check_mixed(As, g, nev, tol, exact_vals, exact_space, order):
    """order(values) sorts the wanted end first."""
    assert g["reason"] == S.CONVERGED_TOL and g["nconv"] >= nev, (g["reason"], g["nconv"], g["stats"])
    ex = np.asarray(exact_vals)
    want = ex[order(ex)][:nev]
    got = g["evals"][:nev]
    assert H.eig_set_match(g["evals"], ex, 0) < 1e-10
    # the distinct values found are the leading distinct values of the spectrum: none skipped
    got_d = np.array([lam for lam, _ in H.clusters(got[order(got)], 1e-9)])
    ex_d = np.array([lam for lam, _ in H.clusters(ex[order(ex)][: 4 * nev], 1e-9)])
    np.testing.assert_allclose(got_d, ex_d[: len(got_d)], rtol=1e-10, atol=0)
    complete = bool(np.allclose(np.sort(got), np.sort(want), rtol=1e-10, atol=0))
    from oracle import residual

    res = np.array([residual(As, g["X"][:, i], g["evals"][i]) for i in range(g["nconv"])])
    assert res[:nev].max() <= tol, res.max()
    np.testing.assert_allclose(g["err"], res, rtol=1e-6, atol=1e-15)
    assert np.abs(g["X"].T @ g["X"] - np.eye(g["nconv"])).max() < 1e-12
    spectrum = np.unique(ex)
    worst = 0.0
    for i in range(nev):
        lam = g["evals"][i]
        others = spectrum[np.abs(spectrum - lam) > 1e-9 * abs(lam)]
        gap = np.abs(others - lam).min()
        s = H.max_subspace_sine(g["X"][:, [i]], exact_space(lam))
        assert s <= max(1.01 * res[i] * abs(lam) / gap, 1e-8), (lam, s)
        worst = max(worst, s)
    return {"max_rel_residual": float(res[:nev].max()), "max_sine_vs_exact": worst, "multiplicities_complete": complete}


def oracle_errors(g, o, nev):
    """Per-eigenpair relative error of the mixed eigenvalues against the FP64 oracle's (sorted)."""
    a = np.sort(g["evals"][:nev])
    b = np.sort(o.evals[:nev])
    m = min(len(a), len(b))
    return (np.abs(a[:m] - b[:m]) / np.abs(b[:m])).tolist()


LARGEST = lambda e: np.argsort(-np.asarray(e), kind="stable")  # noqa: E731
SMALLEST = lambda e: np.argsort(np.asarray(e), kind="stable")  # noqa: E731
MAGNITUDE = lambda e: np.argsort(-np.abs(np.asarray(e)), kind="stable")  # noqa: E731


def test_mixed_2d_laplacian_100(oracle_mod):
    """2-D Laplacian 100x100, nev=10 largest magnitude, ncv=32, tol=1e-8, mixed form."""
    csr = P.laplacian_2d(100)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 0)
    g = mixed_solve(csr, v0, 10, 32, S.LARGEST_MAGNITUDE)
    As = P.to_scipy(csr)
    rep = check_mixed(As, g, 10, 1e-8, P.laplacian_2d_eigs(100), lambda lam: P.laplacian_2d_eigenspace(lam, 100),
                      MAGNITUDE)
    o = oracle_mod.eps_solve(As, v0, nev=10, ncv=32, which=oracle_mod.LARGEST_MAGNITUDE)
    _report("mixed_2d_100", oracle_rel_err=oracle_errors(g, o, 10), **rep,
            sweeps=g["stats"]["filter_sweeps"], restarts=g["stats"]["phase1_restarts"])


@pytest.mark.parametrize("N,seed", [(16, 0), (24, 1)])
def test_mixed_3d_laplacian_nev32(oracle_mod, N, seed):
    """3-D 7-point Laplacian, nev=32 largest real, ncv=80: the true top 32 with multiplicities."""
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, seed)
    g = mixed_solve(csr, v0, 32, 80, S.LARGEST_REAL)
    As = P.to_scipy(csr)
    rep = check_mixed(As, g, 32, 1e-8, P.laplacian_3d_eigs(N), lambda lam: P.laplacian_3d_eigenspace(lam, N),
                      LARGEST)
    o = oracle_mod.eps_solve(As, v0, nev=32, ncv=80, which=oracle_mod.LARGEST_REAL)
    _report(f"mixed_3d_{N}", oracle_rel_err=oracle_errors(g, o, 32), **rep,
            sweeps=g["stats"]["filter_sweeps"], restarts=g["stats"]["phase1_restarts"])


def _random_sym(n, seed, dense_rows=0):
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    B = sp.random(n, n, density=0.01, random_state=rng, format="csr")
    A = B + B.T + sp.diags(rng.standard_normal(n))
    if dense_rows:
        # a few rows and columns with hundreds of nonzeros: rows outside the 32-wide slices
        R = sp.lil_matrix((n, n))
        for r in rng.choice(n, dense_rows, replace=False):
            cols = rng.choice(n, 300, replace=False)
            v = rng.standard_normal(300) * 0.1
            R[r, cols] = v
        R = R.tocsr()
        A = A + R + R.T
    A = A.tocsr()
    A.sort_indices()
    A.eliminate_zeros()
    return A


@pytest.mark.parametrize("dense_rows", [0, 6])
def test_mixed_random_sparse_vs_dense_eigh(dense_rows):
    """Random symmetric sparse matrices (with and without long rows): the mixed pairs equal dense LAPACK."""
    n = 1200
    A = _random_sym(n, 11, dense_rows)
    csr = (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data)
    v0 = P.start_vector(n, 3)
    ev, W = np.linalg.eigh(A.toarray())

    def space(lam):
        return W[:, np.abs(ev - lam) <= 1e-10 * abs(lam)]

    for which, order in ((S.LARGEST_MAGNITUDE, MAGNITUDE), (S.SMALLEST_REAL, SMALLEST), (S.LARGEST_REAL, LARGEST)):
        g = mixed_solve(csr, v0, 6, 30, which)
        rep = check_mixed(A, g, 6, 1e-8, ev, space, order)
        _report(f"mixed_random_which{which}_dense{dense_rows}", **rep)


def test_mixed_fp32_stored_values():
    """A matrix stored with FP32 values: the operator is the FP32 matrix, solved to 1e-8 in FP64."""
    n = 900
    A = _random_sym(n, 5)
    A.data = A.data.astype(np.float32).astype(np.float64)
    csr = (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float32))
    v0 = P.start_vector(n, 1)
    ev, W = np.linalg.eigh(A.toarray())

    def space(lam):
        return W[:, np.abs(ev - lam) <= 1e-10 * abs(lam)]

    g = mixed_solve(csr, v0, 8, 32, S.LARGEST_REAL, dtype=np.float32)
    check_mixed(A, g, 8, 1e-8, ev, space, LARGEST)


def test_mixed_repeatable():
    """Two mixed solves of the same problem return the same bits."""
    csr = P.laplacian_3d(12)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 2)
    g1 = mixed_solve(csr, v0, 16, 48, S.LARGEST_REAL)
    g2 = mixed_solve(csr, v0, 16, 48, S.LARGEST_REAL)
    assert np.array_equal(g1["evals"], g2["evals"])
    assert np.array_equal(g1["X"], g2["X"])


def test_mixed_rejects_smallest_magnitude():
    csr = P.laplacian_2d(20)
    n = len(csr[0]) - 1
    with pytest.raises(S.B200Error):
        mixed_solve(csr, P.start_vector(n, 0), 4, 16, S.SMALLEST_MAGNITUDE)
