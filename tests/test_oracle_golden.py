"""Pin the CPU oracle against SLEPc's own known answers (CPU only).

The fixtures in tests/golden/ were extracted from the reference test outputs
by tests/golden/make_golden.py.
"""
import numpy as np
import pytest

from slepc_b200 import problems as P
from tests import helpers as H


def test_ex2_golden_digits(oracle_mod):
    """src/eps/tutorials/ex2.c -n 72 -eps_nev 4 -eps_ncv 20 -> output/ex2_1.out."""
    g = H.golden("ex2_1.json")
    A = P.to_scipy(P.laplacian_2d(72))
    for seed in (0, 1, 2):
        r = oracle_mod.eps_solve(A, P.start_vector(A.shape[0], seed), nev=4, ncv=20,
                                 which=oracle_mod.LARGEST_MAGNITUDE)
        assert r.reason == oracle_mod.CONVERGED_TOL
        got = [float("%.5f" % v) for v in r.evals[:4]]
        accepted = [o["values"] for o in g["outputs"].values()]
        assert got in accepted, (got, accepted)
        for i in range(r.nconv):
            assert oracle_mod.residual(A, r.X[:, i], r.evals[i]) <= 1e-8


def laplacian_1d(n):
    """The 1-D Laplacian of src/eps/tests/test2.c (2 on the diagonal, -1 beside it)."""
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i)
                cols.append(j)
                vals.append(v)
    rowptr = np.searchsorted(rows, np.arange(n + 1)).astype(np.int32)
    return rowptr, np.array(cols, dtype=np.int32), np.array(vals)


@pytest.mark.parametrize("lock", [True, False])
def test_eps_test2_golden_both_locking_variants(oracle_mod, lock):
    """src/eps/tests/test2.c -eps_type krylovschur -eps_krylovschur_locking {0 1} -> output/test2_1.out:
    the largest and smallest four eigenvalues of the 1-D Laplacian n=30 at tol 1e-9, in both variants
    (the non-locking one keeps converged pairs in the active subspace, krylovschur.c:295)."""
    g = H.golden("eps_test2.json")
    A = P.to_scipy(laplacian_1d(g["args"]["n"]))
    oracle_mod.set_locking(lock)
    try:
        for which, key in ((oracle_mod.LARGEST_REAL, "largest_real"), (oracle_mod.SMALLEST_REAL, "smallest_real")):
            r = oracle_mod.eps_solve(A, P.start_vector(A.shape[0], 5), nev=4, ncv=19, tol=g["args"]["tol"],
                                     which=which)
            assert r.reason == oracle_mod.CONVERGED_TOL and r.nconv >= 4
            assert [float("%.5f" % v) for v in r.evals[:4]] == g[key]
            for i in range(4):
                assert oracle_mod.residual(A, r.X[:, i], r.evals[i]) <= 1e-9
    finally:
        oracle_mod.set_locking(True)


def test_bv_test2_golden(oracle_mod):
    """src/sys/classes/bv/tests/test2.c: CGS orthogonality and the ones-vector norm 2.50931."""
    g = H.golden("bv_test2.json")
    X = H.bv_test2_fixture(g["n"], g["k"])
    for j in range(g["k"]):
        _, nrm, _ = oracle_mod.bv_orthogonalize_column(X, j)
        X[:, j] *= 1.0 / nrm
    M = X.T @ X - np.eye(g["k"])
    assert np.abs(M).sum(axis=0).max() < 100 * np.finfo(float).eps
    _, _, nrm, _ = oracle_mod.bv_orthogonalize_vec(X, g["k"], np.ones(g["n"]))
    assert float("%.5f" % nrm) == pytest.approx(g["norm_ones_after_orth"], abs=0)


def test_ds_test2_golden(oracle_mod):
    """src/sys/classes/ds/tests/test2.c: DSHEP Toeplitz eigenvalues, rnorm of the 3rd vector."""
    g = H.golden("ds_test2.json")
    wr, Q = oracle_mod.ds_hep_dense(H.ds_test2_matrix(g["n"]), oracle_mod.LARGEST_MAGNITUDE, ld=g["ld"])
    assert [float("%.5f" % v) for v in wr] == g["eigenvalues"]
    assert float("%.3f" % abs(Q[g["n"] - 1, 2])) == g["rnorm_3rd"]
    assert float("%.3f" % np.linalg.norm(Q[:, 0])) == g["norm_1st"]


def test_bv_test1_multinplace_golden(oracle_mod):
    """src/sys/classes/bv/tests/test1.c: BVMultInPlace(X,Q,1,l) then BVScale(X,2)."""
    g = H.golden("bv_test1.json")
    X, _, Q = H.bv_test1_fixture()
    oracle_mod.bv_multinplace(X, 0, g["k"], Q, 1, g["l"])
    X *= 2.0
    np.testing.assert_array_equal(X.T, np.array(g["X_after_multinplace_scale2"]))
    assert float("%g" % np.linalg.norm(X[:, 0])) == g["norm2_X0"]
    assert float("%g" % np.linalg.norm(X)) == g["norm_fro"]


def test_oracle_2d_spectrum_against_analytic(oracle_mod):
    """Converged values lie on the analytic 2-D Laplacian spectrum to 1e-10."""
    A = P.to_scipy(P.laplacian_2d(30, 31))
    r = oracle_mod.eps_solve(A, P.start_vector(A.shape[0], 3), nev=8, ncv=24, which=oracle_mod.LARGEST_REAL)
    ex = P.laplacian_2d_eigs(30, 31)
    assert r.nconv >= 8
    assert H.eig_set_match(r.evals, ex, 0) < 1e-10


def test_oracle_dense_check_small(oracle_mod):
    """Small random symmetric sparse matrix: compare with dense LAPACK eigh."""
    rng = np.random.default_rng(5)
    n = 300
    import scipy.sparse as sp

    B = sp.random(n, n, density=0.02, random_state=rng, format="csr")
    A = (B + B.T + sp.diags(rng.standard_normal(n))).tocsr()
    A.sort_indices()
    r = oracle_mod.eps_solve(A, P.start_vector(n, 1), nev=6, ncv=30, which=oracle_mod.LARGEST_MAGNITUDE)
    ev = np.linalg.eigvalsh(A.toarray())
    top = ev[np.argsort(-np.abs(ev))][:6]
    assert r.nconv >= 6
    np.testing.assert_allclose(np.sort(r.evals[:6]), np.sort(top), rtol=1e-10)


def test_oracle_sample_mode_stops(oracle_mod):
    A = P.to_scipy(P.laplacian_2d(40))
    r = oracle_mod.eps_solve(A, P.start_vector(A.shape[0], 0), nev=10, ncv=32,
                             which=oracle_mod.LARGEST_MAGNITUDE, max_restarts=2)
    assert r.restarts == 2 and r.reason == oracle_mod.ITERATING


@pytest.mark.parametrize("block", ["chol", "svqb"])
def test_bv_test11_block_orthogonalization_golden(oracle_mod, block):
    """src/sys/classes/bv/tests/test11.c with -bv_orthog_block chol / svqb (-resid for test11_6):
    columns [0,l) and then [l,k) orthogonalized, every check the expected output lists below
    100 eps.  (Gram-Schmidt is pinned by test2; the TSQR types by tests/test_gpu_tsqr.py.)"""
    g = H.golden("bv_test11.json")
    eps = np.finfo(float).eps
    t = {"chol": oracle_mod.ORTHOG_BLOCK_CHOL, "svqb": oracle_mod.ORTHOG_BLOCK_SVQB}[block]
    for name, o in g["outputs"].items():
        assert block in g["block_types"][name]
        n, l, k = o["n"], o["l"], o["k"]
        X = H.bv_test2_fixture(n, k)  # test11.c:75-91 fills X as test2.c does
        Y = np.asfortranarray(X.copy())
        R1 = oracle_mod.bv_orthogonalize_block(Y, 0, l, t)
        R2 = oracle_mod.bv_orthogonalize_block(Y, l, k, t)
        R = np.zeros((k, k))
        R[:l, :l] = R1[:l, :l]
        R[:, l:] = R2[:, l:]
        M = Y.T @ Y - np.eye(k)
        checks = {"Level of orthogonality of Q1": np.linalg.norm(M[:l, :l]),
                  "Level of orthogonality of Q2": np.linalg.norm(M[l:, l:]),
                  "Level of orthogonality of Q": np.linalg.norm(M)}
        if o["resid"]:
            checks["Residual ||X1-Q1*R11||"] = np.linalg.norm(X[:, :l] - Y[:, :l] @ R[:l, :l])
            checks["Residual ||X-Q*R||"] = np.linalg.norm(X - Y @ R)
        assert sorted(checks) == sorted(o["below_100eps"])
        for label in o["below_100eps"]:
            assert checks[label] < 100 * eps, (name, label, checks[label] / eps)
