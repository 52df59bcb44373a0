"""End-to-end parity of the GPU Krylov-Schur solve with the CPU oracle.

Criteria (FP64 throughout):
  * every converged eigenvalue lies on the exact spectrum (analytic for the
    Laplacians, dense LAPACK otherwise) to 1e-10 relative, and the distinct
    eigenvalues of the GPU run and of the oracle agree to 1e-10 inside the
    window both runs cover;
  * every residual ||Ax - lambda x|| / |lambda| is <= tol, computed in FP64 on the
    host by the oracle and on the device by EPSComputeError;
  * every eigenvector lies in the exact eigenspace within the Davis-Kahan
    bound (residual / gap, floor 1e-8), and where both runs found a multiple
    eigenvalue with its full multiplicity the two eigenspaces coincide within
    the sum of their bounds (floor 1e-8).
Single-vector Krylov-Schur finds the copies of a multiple eigenvalue only
through rounding, so two correct runs can return different multiplicities
(and then a different last eigenvalue); the checks compare eigenspaces per
cluster against the exact eigenspace, not vectors per index.
"""
import json
import os

import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P
from tests import helpers as H

pytestmark = pytest.mark.gpu


def gpu_solve(csr, v0, nev, ncv, which, tol=1e-8, max_restarts=0, lock=True):
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setDimensions(nev, ncv)
    E.setKrylovSchurLocking(lock)
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


def _report(name, **kv):
    """Append measured parity figures to $PARITY_REPORT (JSON lines) when set."""
    path = os.environ.get("PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"test": name, **kv}) + "\n")


def _distinct(vals, rtol=1e-9):
    return np.array([lam for lam, _ in H.clusters(np.sort(vals)[::-1], rtol)])


def check_parity(csr, g, o, oracle_mod, tol, exact_vals, exact_space, key, nev, compare_sets=True):
    """GPU result g vs oracle result o.  exact_space(lam) returns an orthonormal basis of the
    exact eigenspace; key(lam) is larger for the eigenvalues wanted first."""
    As = P.to_scipy(csr)
    assert g["reason"] == S.CONVERGED_TOL and o.reason == oracle_mod.CONVERGED_TOL
    # (1) every computed value lies on the exact spectrum
    assert H.eig_set_match(g["evals"], exact_vals, 0) < 1e-10
    assert H.eig_set_match(o.evals, exact_vals, 0) < 1e-10
    # (2) the distinct values of the requested pairs agree inside the window both runs cover
    if compare_sets:
        gv, ov = g["evals"][:nev], o.evals[:nev]
        thr = max(key(gv).min(), key(ov).min())
        thr -= 1e-9 * abs(thr)  # the two runs compute the cut-off eigenvalue to rounding, not bit for bit
        dg = _distinct(gv[key(gv) >= thr])
        do = _distinct(ov[key(ov) >= thr])
        assert H.eig_set_match(dg, do, 0) < 1e-10 and H.eig_set_match(do, dg, 0) < 1e-10, (dg, do)
    # (3) residuals in FP64 on the host, and the device's EPSComputeError agrees
    res = np.array([oracle_mod.residual(As, g["X"][:, i], g["evals"][i]) for i in range(g["nconv"])])
    assert res.max() <= tol, res.max()
    np.testing.assert_allclose(g["err"], res, rtol=1e-6, atol=1e-15)
    # (4) orthonormal basis
    assert np.abs(g["X"].T @ g["X"] - np.eye(g["nconv"])).max() < 1e-12
    # (5) each eigenvector inside the exact eigenspace within the Davis-Kahan bound
    spectrum = np.unique(np.asarray(exact_vals))
    worst_exact, worst_oracle, bound_min = 0.0, 0.0, np.inf
    for i in range(g["nconv"]):
        lam = g["evals"][i]
        others = spectrum[np.abs(spectrum - lam) > 1e-9 * abs(lam)]
        gap = np.abs(others - lam).min()
        bound = res[i] * abs(lam) / gap
        s_ex = H.max_subspace_sine(g["X"][:, [i]], exact_space(lam))
        assert s_ex <= max(1.01 * bound, 1e-8), (lam, s_ex, bound)
        worst_exact = max(worst_exact, s_ex)
    # (6) clusters found with the full multiplicity by both runs: the two eigenspaces coincide
    for lam, ig in H.clusters(g["evals"], 1e-9):
        io = np.where(np.abs(o.evals - lam) <= 1e-9 * abs(lam))[0]
        mult = exact_space(lam).shape[1]
        if len(ig) == len(io) == mult:
            others = spectrum[np.abs(spectrum - lam) > 1e-9 * abs(lam)]
            gap = np.abs(others - lam).min()
            bound = 2 * tol * abs(lam) / gap
            s = H.max_subspace_sine(g["X"][:, ig], o.X[:, io])
            assert s <= max(bound, 1e-8), (lam, s, bound)
            worst_oracle = max(worst_oracle, s)
            bound_min = min(bound_min, bound)
    return {"max_sine_vs_exact": worst_exact, "max_sine_vs_oracle": worst_oracle,
            "max_rel_residual": float(res.max()), "gpu_nconv": g["nconv"], "oracle_nconv": o.nconv,
            "gpu_its": g["its"], "oracle_its": o.its}


LR = lambda e: np.asarray(e)  # noqa: E731
LM = lambda e: np.abs(np.asarray(e))  # noqa: E731
SR = lambda e: -np.asarray(e)  # noqa: E731


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
    rep = check_parity(csr, g, o, oracle_mod, 1e-8, P.laplacian_2d_eigs(72),
                       lambda lam: P.laplacian_2d_eigenspace(lam, 72), LM, 4)
    _report("ex2_72", **rep)
    assert abs(g["its"] - o.its) <= 2


def test_config1_2d_laplacian_100(oracle_mod):
    """2-D 5-point Laplacian 100x100, nev=10 largest magnitude, ncv=32, tol=1e-8."""
    csr = P.laplacian_2d(100)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, 0)
    g = gpu_solve(csr, v0, 10, 32, S.LARGEST_MAGNITUDE)
    o = oracle_mod.eps_solve(P.to_scipy(csr), v0, nev=10, ncv=32, which=oracle_mod.LARGEST_MAGNITUDE)
    assert g["nconv"] >= 10
    rep = check_parity(csr, g, o, oracle_mod, 1e-8, P.laplacian_2d_eigs(100),
                       lambda lam: P.laplacian_2d_eigenspace(lam, 100), LM, 10)
    _report("config1_2d_100", **rep)


@pytest.mark.parametrize("N,seed", [(16, 0), (24, 1)])
def test_3d_laplacian_nev32_ncv80(oracle_mod, N, seed):
    """The 3-D 7-point Laplacian workload (nev=32 largest real, ncv=80) on small grids."""
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    v0 = P.start_vector(n, seed)
    g = gpu_solve(csr, v0, 32, 80, S.LARGEST_REAL)
    o = oracle_mod.eps_solve(P.to_scipy(csr), v0, nev=32, ncv=80, which=oracle_mod.LARGEST_REAL)
    assert g["nconv"] >= 32
    rep = check_parity(csr, g, o, oracle_mod, 1e-8, P.laplacian_3d_eigs(N),
                       lambda lam: P.laplacian_3d_eigenspace(lam, N), LR, 32)
    _report(f"3d_{N}", **rep)


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
    ev, W = np.linalg.eigh(A.toarray())

    def space(lam):
        return W[:, np.abs(ev - lam) <= 1e-10 * abs(lam)]

    for which, order, key in ((S.LARGEST_MAGNITUDE, lambda e: -np.abs(e), LM), (S.SMALLEST_REAL, lambda e: e, SR),
                              (S.LARGEST_REAL, lambda e: -e, LR)):
        g = gpu_solve(csr, v0, 6, 30, which)
        top = ev[np.argsort(order(ev), kind="stable")][:6]
        np.testing.assert_allclose(g["evals"][:6], top, rtol=1e-10)
        o = oracle_mod.eps_solve(A, v0, nev=6, ncv=30, which=which)
        # the GPU's six pairs equal dense LAPACK's (checked above); the oracle may lock a smaller
        # eigenvalue of this clustered spectrum first, so its set is not compared
        rep = check_parity(csr, g, o, oracle_mod, 1e-8, ev, space, key, 6, compare_sets=False)
        _report(f"random_sparse_which{which}", **rep)


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


def test_zero_initial_vector_falls_back_to_a_random_start(oracle_mod):
    """BVInsertVecs drops a zero initial vector (bvfunc.c:331-374), so EPSGetStartVector draws a
    random one (epssolve.c:852): the solve proceeds, from the same random vector as the oracle."""
    csr = P.laplacian_2d(20)
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(2, 10)
    E.setInitialSpace(np.zeros(A.n))
    E.solve()
    assert E.getConvergedReason() == S.CONVERGED_TOL and E.getConverged() >= 2
    ref = oracle_mod.eps_solve(P.to_scipy(csr), np.zeros(A.n), nev=2, ncv=10)
    assert E.getIterationNumber() == ref.its
    np.testing.assert_allclose([E.getEigenvalue(i) for i in range(2)], ref.evals[:2], rtol=1e-10)


def test_invariant_subspace_start_vector_still_converges():
    """A start vector inside a 3-dimensional invariant subspace of a diagonal matrix: the Krylov space is
    exhausted after 3 steps, the refined Gram-Schmidt continues from rounding residue or a random restart
    (EPSGetStartVector, epssolve.c:841), and the solver still converges to the right pairs."""
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
    exact = np.sort(P.laplacian_3d_eigs(N))[::-1][:200]
    assert H.eig_set_match(g["evals"], exact, 0) < 1e-10
    assert g["err"].max() <= 1e-8
    XtX = g["X"].T @ g["X"]
    assert np.abs(XtX - np.eye(g["nconv"])).max() < 1e-12
    spectrum = np.unique(exact)
    worst = 0.0
    for i in range(g["nconv"]):
        lam = g["evals"][i]
        gap = np.abs(spectrum[np.abs(spectrum - lam) > 1e-9 * lam] - lam).min()
        s = H.max_subspace_sine(g["X"][:, [i]], P.laplacian_3d_eigenspace(lam, N))
        assert s <= max(1.01 * g["err"][i] * lam / gap, 1e-8), (lam, s)
        worst = max(worst, s)
    _report("config2_128", max_sine_vs_exact=worst, max_rel_residual=float(g["err"].max()), gpu_nconv=g["nconv"],
            gpu_its=g["its"])


FIXTURE_128 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "laplacian3d_128_oracle.json")


@pytest.mark.skipif(not os.path.exists(FIXTURE_128), reason="full-size oracle fixture not generated")
def test_config2_full_size_vs_oracle():
    """The 128^3 workload against the oracle's complete solve of the same CSR and start vector
    (tests/golden/make_laplacian3d_fixture.py):
      * restarts within +-2 of the oracle's;
      * every residual of both runs <= 1e-8 (FP64);
      * the distinct eigenvalues agree to 1e-10 inside the window both runs cover;
      * per eigenvalue cluster, each run's eigenvectors lie in the exact eigenspace within the
        Davis-Kahan bound (residual * lambda / gap); where both runs found the full multiplicity,
        the two computed eigenspaces then coincide within the sum of the two bounds (both span the
        whole exact eigenspace up to their components outside it, which the fixture stores);
        where a run found fewer copies, the angle between the two runs' spans inside the exact
        eigenspace is reported, not asserted (single-vector Krylov picks them through rounding)."""
    with open(FIXTURE_128) as f:
        fx = json.load(f)
    N = 128
    csr = P.laplacian_3d(N)
    n = len(csr[0]) - 1
    g = gpu_solve(csr, P.start_vector(n, 0), 32, 80, S.LARGEST_REAL)
    assert g["reason"] == S.CONVERGED_TOL and g["nconv"] >= 32
    assert abs(g["its"] - fx["its"]) <= 2, (g["its"], fx["its"])
    assert g["err"].max() <= 1e-8
    assert max(p["residual"] for p in fx["pairs"]) <= 1e-8
    gv = g["evals"]
    ov = np.array([p["eigenvalue"] for p in fx["pairs"]])
    lo = max(gv.min(), ov.min())
    gd = np.array([lam for lam, _ in H.clusters(np.sort(gv[gv >= lo * (1 - 1e-12)])[::-1], 1e-9)])
    od = np.array([lam for lam, _ in H.clusters(np.sort(ov[ov >= lo * (1 - 1e-12)])[::-1], 1e-9)])
    assert len(gd) == len(od), (gd, od)
    np.testing.assert_allclose(gd, od, rtol=1e-10, atol=0)
    spectrum = np.unique(np.sort(P.laplacian_3d_eigs(N))[::-1][:400])
    clusters = []
    for lam in gd:
        gi = np.where(np.abs(gv - lam) <= 1e-9 * lam)[0]
        oi = np.where(np.abs(ov - lam) <= 1e-9 * lam)[0]
        B = P.laplacian_3d_eigenspace(lam, N)
        d = B.shape[1]
        gap = np.abs(spectrum[np.abs(spectrum - lam) > 1e-9 * lam] - lam).min()
        Cg = B.T @ g["X"][:, gi]
        out_g = np.linalg.norm(g["X"][:, gi] - B @ Cg, 2)
        out_o = max(fx["pairs"][i]["outside_norm"] for i in oi)
        dk_g = max(1.01 * max(g["err"][i] for i in gi) * lam / gap, 1e-8)
        dk_o = max(1.01 * max(fx["pairs"][i]["residual"] for i in oi) * lam / gap, 1e-8)
        assert out_g <= dk_g and out_o <= dk_o, (lam, out_g, dk_g, out_o, dk_o)
        Co = np.array([fx["pairs"][i]["coefficients"] for i in oi]).T
        inner = H.max_subspace_sine(Cg, Co) if len(gi) <= len(oi) else H.max_subspace_sine(Co, Cg)
        full = len(gi) == len(oi) == d
        if full:
            assert inner <= 1e-6 and out_g + out_o <= dk_g + dk_o
        clusters.append({"eigenvalue": float(lam), "dim": d, "gpu_copies": int(len(gi)), "oracle_copies": int(len(oi)),
                         "sine_bound": float(out_g + out_o + inner), "davis_kahan": float(dk_g + dk_o),
                         "full_multiplicity_both": bool(full)})
    _report("config2_128_vs_oracle", gpu_its=g["its"], oracle_its=fx["its"], oracle_wall_s=fx["wall_s"],
            oracle_threads=fx["threads"], distinct_window=len(gd), clusters=clusters,
            max_eig_rel_diff=float(np.max(np.abs(gd - od) / od)))


@pytest.mark.parametrize("lock", [True, False])
def test_eps_test2_golden_both_locking_variants(oracle_mod, lock):
    """src/eps/tests/test2.c -eps_type krylovschur -eps_krylovschur_locking {0 1} (output/test2_1.out):
    1-D Laplacian n=30, nev=4, tol=1e-9, largest and smallest real -- the reference's digits in both
    variants, and the oracle's eigenvalues (1e-10) and iteration count (+-2) with the same variant."""
    from tests.test_oracle_golden import laplacian_1d

    g = H.golden("eps_test2.json")
    csr = laplacian_1d(g["args"]["n"])
    A = P.to_scipy(csr)
    v0 = P.start_vector(A.shape[0], 5)
    oracle_mod.set_locking(lock)
    try:
        for which, owhich, key in ((S.LARGEST_REAL, oracle_mod.LARGEST_REAL, "largest_real"),
                                   (S.SMALLEST_REAL, oracle_mod.SMALLEST_REAL, "smallest_real")):
            gg = gpu_solve(csr, v0, 4, 19, which, tol=g["args"]["tol"], lock=lock)
            o = oracle_mod.eps_solve(A, v0, nev=4, ncv=19, tol=g["args"]["tol"], which=owhich)
            assert gg["reason"] == S.CONVERGED_TOL and gg["nconv"] >= 4
            assert [float("%.5f" % v) for v in gg["evals"][:4]] == g[key]
            np.testing.assert_allclose(gg["evals"][:4], o.evals[:4], rtol=1e-10)
            assert abs(gg["its"] - o.its) <= 2
            assert gg["err"][:4].max() <= 1e-9
    finally:
        oracle_mod.set_locking(True)


def test_nonlocking_2d_laplacian_vs_oracle(oracle_mod):
    """The non-locking variant on the 2-D Laplacian 60x60 (nev 8, ncv 20, several restarts) against the
    oracle's non-locking run on the same start vector."""
    csr = P.laplacian_2d(60)
    A = P.to_scipy(csr)
    v0 = P.start_vector(A.shape[0], 1)
    g = gpu_solve(csr, v0, 8, 20, S.LARGEST_REAL, tol=1e-9, lock=False)
    oracle_mod.set_locking(False)
    try:
        o = oracle_mod.eps_solve(A, v0, nev=8, ncv=20, tol=1e-9, which=oracle_mod.LARGEST_REAL)
    finally:
        oracle_mod.set_locking(True)
    assert g["reason"] == S.CONVERGED_TOL and o.its > 3
    assert abs(g["its"] - o.its) <= 2
    np.testing.assert_allclose(g["evals"][:8], o.evals[:8], rtol=1e-10)
    assert H.eig_set_match(g["evals"], P.laplacian_2d_eigs(60), 0) < 1e-10
    assert g["err"][:8].max() <= 1e-9


def test_nonlocking_rejects_restricted_mpd():
    """krylovschur.c:116: the non-locking variant does not take an mpd below ncv."""
    csr = P.laplacian_2d(30)
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(20, 30, 12)
    E.setKrylovSchurLocking(False)
    assert not E.getKrylovSchurLocking()
    with pytest.raises(S.B200Error) as ei:
        E.solve()
    assert ei.value.status == 11
    E.destroy()
    A.destroy()


def test_monitor_once_per_restart(tmp_path):
    """EPSMonitorSet: the callback runs once per outer iteration with the iteration number, the
    converged count (nondecreasing with locking) and the current estimates; the JSON-lines monitor
    writes the same iterations; a monitor that returns true aborts the solve."""
    import json as _json

    csr = P.laplacian_2d(60)
    n = len(csr[0]) - 1
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(8, 20)
    E.setTolerances(1e-9)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    E.setInitialSpace(P.start_vector(n, 1))
    seen = []
    E.setMonitor(lambda its, nconv, eigr, errest: seen.append((its, nconv, eigr[nconv:nconv + 1].copy(), len(errest))))
    path = tmp_path / "monitor.jsonl"
    E.setMonitorJSONL(str(path))
    E.solve()
    its = E.getIterationNumber()
    assert [s[0] for s in seen] == list(range(1, its + 1))
    assert all(a[1] <= b[1] for a, b in zip(seen, seen[1:]))
    assert seen[-1][1] == E.getConverged()
    lines = [_json.loads(x) for x in path.read_text().splitlines()]
    assert [d["its"] for d in lines] == list(range(1, its + 1))
    assert lines[-1]["nconv"] == E.getConverged() and len(lines[-1]["errest"]) == lines[-1]["nest"]
    assert all(a["ms"] <= b["ms"] and a["gs_bytes"] <= b["gs_bytes"] for a, b in zip(lines, lines[1:]))
    # a monitor asking to stop
    E.cancelMonitor()
    E.setMonitor(lambda its, nconv, eigr, errest: its >= 2)
    with pytest.raises(S.B200Error) as ei:
        E.solve()
    assert ei.value.status == 7
    E.cancelMonitor()
    # the mixed form reports once per sweep
    seen.clear()
    E.setMonitor(lambda its, nconv, eigr, errest: seen.append((its, nconv)))
    E.setPrecision(S.EPS.Precision.MIXED)
    E.solve()
    st = E.getStats()
    assert [s[0] for s in seen] == list(range(1, st["phase1_restarts"] + st["filter_sweeps"] + 1))
    assert seen[-1][1] >= 8
    E.destroy()
    A.destroy()
