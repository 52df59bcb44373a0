"""CPU checks of the LOBPCG oracle and of the anisotropic-diffusion generator."""
import numpy as np
import pytest

from slepc_b200 import problems as P


def test_diffusion_generator():
    csr, kappa, corr = P.diffusion_problem(40, 7)
    A = P.to_scipy(csr)
    assert 0.05 <= corr <= 0.2
    assert abs(A - A.T).max() == 0.0
    assert np.all(np.linalg.eigvalsh(A.toarray()) > 0)
    g = np.log(kappa)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12
    # constant kappa: the 5-point Laplacian with Dirichlet faces at half a cell
    c = P.to_scipy(P.diffusion_fv(np.ones((6, 6))))
    assert c[0, 0] == 6.0 and c[7, 7] == 4.0 and c[0, 1] == -1.0 and c[0, 6] == -1.0
    # deterministic in the seed
    csr2, _, _ = P.diffusion_problem(40, 7)
    assert all(np.array_equal(a, b) for a, b in zip(csr, csr2))


@pytest.mark.parametrize("which", ["smallest", "largest"])
def test_oracle_lobpcg_vs_dense(oracle_mod, which):
    oracle_mod.set_threads(1)
    csr, _, _ = P.diffusion_problem(24, 2)
    A = P.to_scipy(csr)
    w = oracle_mod.SMALLEST_REAL if which == "smallest" else oracle_mod.LARGEST_REAL
    r = oracle_mod.lobpcg(A, 6, bs=6, pc="jacobi", which=w, tol=1e-9, max_it=5000)
    d = np.linalg.eigvalsh(A.toarray())
    exact = d[:6] if which == "smallest" else d[::-1][:6]
    assert r.reason == oracle_mod.CONVERGED_TOL
    np.testing.assert_allclose(r.evals[:6], exact, rtol=1e-11)
    for i in range(6):
        assert np.linalg.norm(A @ r.X[:, i] - r.evals[i] * r.X[:, i]) / abs(r.evals[i]) < 1e-9
    assert np.abs(r.X[:, :6].T @ r.X[:, :6] - np.eye(6)).max() < 1e-12


@pytest.mark.parametrize("l", [0, 4])
def test_oracle_block_orthogonalization(oracle_mod, l):
    """BVOrthogonalize with the Cholesky and SVQB block types: V_in = V_out R, V_out orthonormal,
    the leading columns untouched; Cholesky gives the Q of a QR factorisation with R's diagonal
    positive (numpy's Householder QR with the signs fixed), SVQB a symmetric-polar-like basis."""
    rng = np.random.default_rng(3)
    n, k = 700, 12
    V0 = rng.standard_normal((n, k))
    if l:
        V0[:, :l] = np.linalg.qr(V0[:, :l])[0]
    for t in (oracle_mod.ORTHOG_BLOCK_CHOL, oracle_mod.ORTHOG_BLOCK_SVQB):
        V = np.asfortranarray(V0.copy())
        R = oracle_mod.bv_orthogonalize_block(V, l, k, t)
        assert np.array_equal(V[:, :l], V0[:, :l])
        assert np.abs(V.T @ V - np.eye(k)).max() < 1e-13
        assert np.abs(V @ R[:, l:] - V0[:, l:]).max() < 1e-12 * np.abs(V0).max() * n ** 0.5
        if t == oracle_mod.ORTHOG_BLOCK_CHOL:
            assert np.all(np.tril(R[l:, l:], -1) == 0.0) and np.all(np.diag(R)[l:] > 0)
            # the block after one Gram-Schmidt pass against the leading columns, then QR
            W = V0[:, l:] - V0[:, :l] @ (V0[:, :l].T @ V0[:, l:])
            Q, Rq = np.linalg.qr(W)
            Q = Q * np.sign(np.diag(Rq))
            assert np.abs(V[:, l:] - Q).max() < 1e-12


@pytest.mark.parametrize("block", ["chol", "svqb"])
def test_oracle_lobpcg_block_types_vs_dense(oracle_mod, block):
    """LOBPCG with Cholesky / SVQB block orthogonalization (hard locking, nev > bs - guard)
    converges to the dense spectrum, like the Gram-Schmidt default."""
    oracle_mod.set_threads(1)
    csr, _, _ = P.diffusion_problem(24, 2)
    A = P.to_scipy(csr)
    t = {"chol": oracle_mod.ORTHOG_BLOCK_CHOL, "svqb": oracle_mod.ORTHOG_BLOCK_SVQB}[block]
    r = oracle_mod.lobpcg(A, 10, bs=4, pc="jacobi", which=oracle_mod.SMALLEST_REAL, tol=1e-9, max_it=5000,
                          orthog_block=t)
    g = oracle_mod.lobpcg(A, 10, bs=4, pc="jacobi", which=oracle_mod.SMALLEST_REAL, tol=1e-9, max_it=5000)
    d = np.linalg.eigvalsh(A.toarray())
    assert r.reason == oracle_mod.CONVERGED_TOL
    np.testing.assert_allclose(r.evals[:10], d[:10], rtol=1e-11)
    assert abs(r.its - g.its) <= max(3, g.its // 10), (r.its, g.its)
    for i in range(10):
        assert np.linalg.norm(A @ r.X[:, i] - r.evals[i] * r.X[:, i]) / abs(r.evals[i]) < 1e-9
