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
