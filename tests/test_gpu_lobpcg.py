"""GPU parity of the LOBPCG solver (EPSLOBPCG) against the CPU oracle and dense LAPACK.

Cases cover the smallest and the largest end, the Jacobi and the identity
preconditioner, soft locking only and hard locking with constraint vectors
(nev > bs - guard), locking switched off, and a block initial space.
Eigenvalues agree with the oracle to 1e-10 relative and with dense eigh;
iteration counts agree within 2 (the two sides round the Gram matrices in a
different order); every residual ||Ax - lambda x|| / |lambda| is checked in
FP64 on the host; eigenvectors lie in the exact eigenspaces within the
Davis-Kahan bound.
"""
import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P

pytestmark = pytest.mark.gpu


def _gpu_lobpcg(csr, nev, bs, pc, which, tol=1e-8, lock=True, X0=None, max_it=5000):
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setType(S.EPS.Type.LOBPCG)
    E.setDimensions(nev)
    E.setLOBPCGBlockSize(bs)
    E.setLOBPCGLocking(lock)
    E.setPreconditioner({"jacobi": S.EPS.PCType.JACOBI, "none": S.EPS.PCType.NONE}[pc])
    E.setTolerances(tol, max_it)
    E.setWhichEigenpairs(which)
    if X0 is not None:
        E.setInitialSpace(X0)
    E.solve()
    k = E.getConverged()
    pairs = [E.getEigenpair(i) for i in range(k)]
    return E, A, np.array([p[0] for p in pairs]), np.array([p[1] for p in pairs]).T


CASES = [
    ("diffusion 32^2, smallest 4, bs 4, Jacobi", lambda: P.diffusion_problem(32, 1)[0], 4, 4, "jacobi",
     S.SMALLEST_REAL, True),
    ("diffusion 32^2, smallest 10, bs 4, hard locking", lambda: P.diffusion_problem(32, 1)[0], 10, 4, "jacobi",
     S.SMALLEST_REAL, True),
    ("laplacian 30x31, largest 6, no preconditioner", lambda: P.laplacian_2d(30, 31), 6, 6, "none",
     S.LARGEST_REAL, True),
    ("diffusion 24^2, smallest 8, locking off", lambda: P.diffusion_problem(24, 3)[0], 8, 8, "jacobi",
     S.SMALLEST_REAL, False),
]


@pytest.mark.parametrize("name,make,nev,bs,pc,which,lock", CASES, ids=[c[0] for c in CASES])
def test_lobpcg_parity_vs_oracle_and_dense(oracle_mod, name, make, nev, bs, pc, which, lock):
    oracle_mod.set_threads(1)
    csr = make()
    As = P.to_scipy(csr)
    E, A, lam, X = _gpu_lobpcg(csr, nev, bs, pc, which, lock=lock)
    ref = oracle_mod.lobpcg(As, nev, bs=bs, pc=pc, which={S.SMALLEST_REAL: oracle_mod.SMALLEST_REAL,
                                                          S.LARGEST_REAL: oracle_mod.LARGEST_REAL}[which],
                            tol=1e-8, max_it=5000, lock=lock)
    assert E.getConvergedReason() == S.CONVERGED_TOL and ref.reason == oracle_mod.CONVERGED_TOL
    assert len(lam) >= nev and ref.nconv >= nev
    assert abs(E.getIterationNumber() - ref.its) <= 2, (E.getIterationNumber(), ref.its)
    np.testing.assert_allclose(lam[:nev], ref.evals[:nev], rtol=1e-10)
    d, Q = np.linalg.eigh(As.toarray())
    exact = d[:nev] if which == S.SMALLEST_REAL else d[::-1][:nev]
    np.testing.assert_allclose(lam[:nev], exact, rtol=1e-10)
    for i in range(nev):
        r = np.linalg.norm(As @ X[:, i] - lam[i] * X[:, i]) / abs(lam[i])
        assert r < 1e-8, (i, r)
        assert abs(E.computeError(i) - r) <= 1e-12 + 1e-6 * r
        # inside the exact eigenspace of lam[i] within the Davis-Kahan bound
        gap = np.min(np.abs(np.delete(d, np.where(np.abs(d - lam[i]) <= 1e-10 * abs(lam[i]))[0]) - lam[i]))
        space = Q[:, np.abs(d - lam[i]) <= 1e-10 * abs(lam[i])]
        sine = np.linalg.norm(X[:, i] - space @ (space.T @ X[:, i]))
        assert sine <= 2 * r * abs(lam[i]) / gap + 1e-12, (i, sine)


def test_lobpcg_block_initial_space_parity(oracle_mod):
    """EPSSetInitialSpace with a block (rough eigenvectors plus noise): the same iterations as the oracle,
    and fewer than from the random start."""
    oracle_mod.set_threads(1)
    csr, _, _ = P.diffusion_problem(32, 5)
    As = P.to_scipy(csr)
    d, Q = np.linalg.eigh(As.toarray())
    rng = np.random.default_rng(0)
    X0 = Q[:, :6] + 1e-3 * rng.standard_normal((As.shape[0], 6))
    E, A, lam, X = _gpu_lobpcg(csr, 6, 6, "jacobi", S.SMALLEST_REAL, X0=X0)
    ref = oracle_mod.lobpcg(As, 6, bs=6, pc="jacobi", which=oracle_mod.SMALLEST_REAL, tol=1e-8, max_it=5000, X0=X0)
    cold = oracle_mod.lobpcg(As, 6, bs=6, pc="jacobi", which=oracle_mod.SMALLEST_REAL, tol=1e-8, max_it=5000)
    assert E.getConvergedReason() == S.CONVERGED_TOL
    assert abs(E.getIterationNumber() - ref.its) <= 2
    assert E.getIterationNumber() < cold.its
    np.testing.assert_allclose(lam[:6], d[:6], rtol=1e-10)


def test_lobpcg_argument_checks():
    csr = P.laplacian_2d(10)
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setType(S.EPS.Type.LOBPCG)
    E.setDimensions(4)
    E.setWhichEigenpairs(S.LARGEST_MAGNITUDE)
    with pytest.raises(S.B200Error):
        E.solve()  # LOBPCG: smallest or largest real only
    E.setWhichEigenpairs(S.SMALLEST_REAL)
    E.setLOBPCGBlockSize(30)
    with pytest.raises(S.B200Error):
        E.solve()  # n = 100 < 5 * bs
    with pytest.raises(S.B200Error):
        E.setLOBPCGRestart(0.05)


@pytest.mark.parametrize("l", [0, 5])
@pytest.mark.parametrize("block", ["chol", "svqb"])
def test_bv_orthogonalize_block_types_vs_oracle(oracle_mod, block, l):
    """BVOrthogonalize with the Cholesky and SVQB block types through the C ABI against the
    oracle on the same columns: the orthonormal block and R agree to 1e-11 (the Gram matrices are
    summed in a different order), V_in = V_out R, the leading columns are untouched."""
    rng = np.random.default_rng(11)
    n, k = 5000, 14
    V0 = rng.standard_normal((n, k))
    if l:
        V0[:, :l] = np.linalg.qr(V0[:, :l])[0]
    tb = {"chol": S.BV.OrthogBlockType.CHOL, "svqb": S.BV.OrthogBlockType.SVQB}[block]
    bv = S.BV().create(n, k)
    bv.setColumns(V0)
    bv.setOrthogonalizationBlock(tb)
    assert bv.getOrthogonalizationBlock() == tb
    bv.setActiveColumns(l, k)
    R = bv.orthogonalize(k)
    V = bv.getColumns(k)
    Vo = np.asfortranarray(V0.copy())
    Ro = oracle_mod.bv_orthogonalize_block(Vo, l, k, {"chol": oracle_mod.ORTHOG_BLOCK_CHOL,
                                                      "svqb": oracle_mod.ORTHOG_BLOCK_SVQB}[block])
    assert np.array_equal(V[:, :l], V0[:, :l])
    assert np.abs(V.T @ V - np.eye(k)).max() < 1e-13
    assert np.abs(V - Vo).max() < 1e-11
    assert np.abs(R[:, l:] - Ro[:, l:]).max() < 1e-11 * np.abs(Ro).max()
    assert np.abs(V @ R[:, l:] - V0[:, l:]).max() < 1e-11


def test_bv_orthog_block_unknown_type_and_breakdown():
    bv = S.BV().create(100, 4)
    with pytest.raises(S.B200Error):
        bv.setOrthogonalizationBlock(7)
    with pytest.raises(S.B200Error):
        bv.setOrthogonalizationBlock(-1)
    # a zero column: SVQB reports a breakdown instead of dividing by zero
    x = np.random.default_rng(0).standard_normal(100)
    bv.setColumns(np.stack([x, np.zeros(100), x + 1, np.ones(100)], axis=1))
    bv.setOrthogonalizationBlock(S.BV.OrthogBlockType.SVQB)
    with pytest.raises(S.B200Error):
        bv.orthogonalize(4)


BLOCK_CASES = [
    ("diffusion 32^2, smallest 10, bs 4, hard locking", lambda: P.diffusion_problem(32, 1)[0], 10, 4, "jacobi",
     S.SMALLEST_REAL),
    ("laplacian 30x31, largest 6, no preconditioner", lambda: P.laplacian_2d(30, 31), 6, 6, "none",
     S.LARGEST_REAL),
]


@pytest.mark.parametrize("block", ["chol", "svqb"])
@pytest.mark.parametrize("name,make,nev,bs,pc,which", BLOCK_CASES, ids=[c[0] for c in BLOCK_CASES])
def test_lobpcg_block_orthogonalization_parity(oracle_mod, name, make, nev, bs, pc, which, block):
    """LOBPCG with -bv_orthog_block chol / svqb: the same iterations (within 2) and eigenvalues
    (1e-10) as the oracle run with the same block type, and the dense spectrum."""
    oracle_mod.set_threads(1)
    csr = make()
    As = P.to_scipy(csr)
    tb = {"chol": S.BV.OrthogBlockType.CHOL, "svqb": S.BV.OrthogBlockType.SVQB}[block]
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setType(S.EPS.Type.LOBPCG)
    E.setDimensions(nev)
    E.setLOBPCGBlockSize(bs)
    E.setPreconditioner({"jacobi": S.EPS.PCType.JACOBI, "none": S.EPS.PCType.NONE}[pc])
    E.setTolerances(1e-8, 5000)
    E.setWhichEigenpairs(which)
    E.setBVOrthogonalizationBlock(tb)
    E.solve()
    lam = np.array([E.getEigenvalue(i) for i in range(E.getConverged())])
    ref = oracle_mod.lobpcg(As, nev, bs=bs, pc=pc, which={S.SMALLEST_REAL: oracle_mod.SMALLEST_REAL,
                                                          S.LARGEST_REAL: oracle_mod.LARGEST_REAL}[which],
                            tol=1e-8, max_it=5000,
                            orthog_block={"chol": oracle_mod.ORTHOG_BLOCK_CHOL,
                                          "svqb": oracle_mod.ORTHOG_BLOCK_SVQB}[block])
    assert E.getConvergedReason() == S.CONVERGED_TOL and ref.reason == oracle_mod.CONVERGED_TOL
    assert abs(E.getIterationNumber() - ref.its) <= 2, (E.getIterationNumber(), ref.its)
    np.testing.assert_allclose(lam[:nev], ref.evals[:nev], rtol=1e-10)
    d = np.linalg.eigvalsh(As.toarray())
    exact = d[:nev] if which == S.SMALLEST_REAL else d[::-1][:nev]
    np.testing.assert_allclose(lam[:nev], exact, rtol=1e-10)
    for i in range(nev):
        assert E.computeError(i) < 1e-8
