"""GPU parity of the batched persistent Krylov-Schur (one launch, one CTA per problem) against the
CPU oracle run problem by problem.

The device solves the projected problem with its own implicit QL iteration instead of LAPACK
dsteqr, so restart decisions can differ in rare cases: iteration counts are compared within 2,
eigenvalues to 1e-10 relative, and the converged eigenvectors are checked for residuals below the
tolerance in FP64 on the host."""
import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P

pytestmark = pytest.mark.gpu


def _batch(nprob, seed, lo, hi):
    ns = P.batch_sizes(nprob, seed, lo, hi)
    B = P.knn_batch(ns, 8, seed)
    v0 = np.concatenate([P.start_vector(int(n), 1000 * seed + p) for p, n in enumerate(ns)])
    return B, v0


def _solve(B, v0, threads, nev=8, ncv=24, tol=1e-8):
    E = S.BatchEPS().create(B.ns, B.rowptr, B.colind, B.vals)
    E.setDimensions(nev, ncv)
    E.setTolerances(tol)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    if v0 is not None:
        E.setInitialVectors(v0)
    E.setThreads(threads)
    E.solve()
    return E


@pytest.mark.parametrize("threads", [128, 256, 512])
def test_batched_parity_vs_oracle(oracle_mod, threads):
    B, v0 = _batch(48, 3, 500, 3000)
    E = _solve(B, v0, threads)
    ev, info, ms = E.getAll()
    oev, oinfo = oracle_mod.eps_solve_batch(B.ns, B.rowptr, B.colind, B.vals, v0, 8, 24, 1e-8,
                                            oracle_mod.LARGEST_REAL, threads=8)
    assert ms > 0
    for p in range(B.nprob):
        assert info[p, 2] == S.CONVERGED_TOL and info[p, 4] == 0
        assert info[p, 0] >= 8 and oinfo[p, 0] >= 8
        assert abs(int(info[p, 1]) - int(oinfo[p, 1])) <= 2, (p, info[p], oinfo[p])
        np.testing.assert_allclose(ev[p, :8], oev[p, :8], rtol=1e-10)
    for p in (0, 7, 31):
        As = P.to_scipy(B.problem(p))
        sol = E.getSolution(p)
        for i in range(8):
            x = E.getEigenvector(p, i)
            r = np.linalg.norm(As @ x - sol["evals"][i] * x) / abs(sol["evals"][i])
            assert r < 2e-8, (p, i, r)
            assert abs(np.linalg.norm(x) - 1.0) < 1e-12


def test_batched_is_deterministic_and_replays_the_graph():
    B, v0 = _batch(40, 4, 500, 2500)
    E = _solve(B, v0, 256)
    ev1, info1, _ = E.getAll()
    E.solve()  # replays the captured graph
    ev2, info2, _ = E.getAll()
    assert np.array_equal(ev1, ev2) and np.array_equal(info1, info2)


def test_batched_random_starts_match_oracle(oracle_mod):
    """No start vectors: every problem starts from the splitmix random column, as the oracle does
    for a dropped zero initial vector."""
    B, _ = _batch(16, 5, 500, 1500)
    E = _solve(B, None, 256)
    ev, info, _ = E.getAll()
    zeros = np.zeros(int(B.ns.sum()))
    oev, oinfo = oracle_mod.eps_solve_batch(B.ns, B.rowptr, B.colind, B.vals, zeros, 8, 24, 1e-8,
                                            oracle_mod.LARGEST_REAL, threads=8)
    for p in range(B.nprob):
        assert info[p, 2] == S.CONVERGED_TOL
        np.testing.assert_allclose(ev[p, :8], oev[p, :8], rtol=1e-10)


def test_batched_autotune_and_arguments():
    B, v0 = _batch(200, 6, 500, 4000)
    E = S.BatchEPS().create(B.ns, B.rowptr, B.colind, B.vals)
    E.setDimensions(8, 24)
    E.setInitialVectors(v0)
    assert E.autotune() in (128, 256, 512)
    E.solve()
    _, info, _ = E.getAll()
    assert np.all(info[:, 2] == S.CONVERGED_TOL)
    with pytest.raises(S.B200Error):
        E.setDimensions(8, 40)  # ncv + 1 > 32
    with pytest.raises(S.B200Error):
        E.setThreads(100)


@pytest.mark.parametrize("threads", [256, 512])
def test_batched_mixed_precision_vs_oracle(oracle_mod, threads):
    """The mixed form: phase 1 on FP32 bases to 1e-6, phase 2 in FP64 from the phase-1 Ritz vectors.
    Eigenvalues equal the FP64 oracle's to 1e-10, residuals in FP64 below the tolerance, both phases
    report their counters."""
    B, v0 = _batch(48, 3, 500, 3000)
    E = S.BatchEPS().create(B.ns, B.rowptr, B.colind, B.vals)
    E.setDimensions(8, 24)
    E.setTolerances(1e-8)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    E.setInitialVectors(v0)
    E.setThreads(threads)
    E.setPrecision(S.EPS.Precision.MIXED, 1e-6)
    E.solve()
    ev, info, ms = E.getAll()
    info1, bytes1 = E.getPhase1()
    oev, oinfo = oracle_mod.eps_solve_batch(B.ns, B.rowptr, B.colind, B.vals, v0, 8, 24, 1e-8,
                                            oracle_mod.LARGEST_REAL, threads=8)
    assert ms > 0 and 0 < bytes1 < E.getBytes()
    for p in range(B.nprob):
        assert info[p, 2] == S.CONVERGED_TOL and info[p, 4] == 0 and info1[p, 4] == 0
        assert info1[p, 0] >= 8 and info[p, 0] >= 8
        np.testing.assert_allclose(ev[p, :8], oev[p, :8], rtol=1e-10)
    assert info1[:, 3].sum() > 0 and info[:, 3].sum() > 0
    for p in (0, 11, 40):
        As = P.to_scipy(B.problem(p))
        sol = E.getSolution(p)
        for i in range(8):
            x = E.getEigenvector(p, i)
            r = np.linalg.norm(As @ x - sol["evals"][i] * x) / abs(sol["evals"][i])
            assert r < 2e-8, (p, i, r)
    E.destroy()
