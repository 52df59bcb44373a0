"""CPU checks of the SVD cross workload: the power-law generator against its
pure-Python restatement, the oracle's transpose and SVD against scipy / dense
LAPACK, and argument rejection of the rectangular-matrix entry points (host
checks that run before any device call)."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from slepc_b200 import problems as P


def test_powerlaw_generator_matches_python_restatement():
    for (m, n, k, alpha, seed) in [(200, 1000, 20, 1.8, 7), (50, 15, 20, 1.8, 1), (80, 300, 5, 2.5, 3)]:
        a = P.powerlaw_rect(m, n, k, alpha, seed)
        b = P.powerlaw_rect_py(m, n, k, alpha, seed)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_powerlaw_generator_structure():
    m, n, k = 5000, 3000, 20
    rowptr, colind, vals = P.powerlaw_rect(m, n, k, 1.8, 0)
    assert vals.dtype == np.float32 and rowptr[-1] == m * k
    rows = colind.reshape(m, k)
    assert np.all(np.diff(rows, axis=1) > 0), "columns sorted and distinct in every row"
    deg = np.bincount(colind, minlength=n)
    assert deg[0] == m and np.all(np.diff(deg[:8]) <= 0)
    assert abs(vals.mean()) < 0.02 and abs(vals.std() - 1.0) < 0.02
    # fewer columns than nnz_row: every column once
    r2, c2, _ = P.powerlaw_rect(10, 7, 20, 1.8, 0)
    assert r2[-1] == 70 and np.array_equal(c2.reshape(10, 7), np.tile(np.arange(7), (10, 1)))


def test_oracle_transpose_matches_scipy(oracle_mod):
    rowptr, colind, vals = P.powerlaw_rect(700, 300, 12, 1.8, 2)
    S = sp.csr_matrix((vals.astype(np.float64), colind, rowptr), shape=(700, 300))
    rt, ct, vt = oracle_mod.csr_transpose(rowptr, colind, S.data, (700, 300))
    T = S.T.tocsr()
    T.sort_indices()
    assert np.array_equal(rt, T.indptr) and np.array_equal(ct, T.indices) and np.array_equal(vt, T.data)


@pytest.mark.parametrize("shape,largest", [((3000, 400), True), ((300, 1600), True), ((600, 80), False)])
def test_oracle_svd_cross_vs_dense(oracle_mod, shape, largest):
    m, n = shape
    if largest:
        rowptr, colind, vals = P.powerlaw_rect(m, n, 20, 1.8, 4)
        S = sp.csr_matrix((vals.astype(np.float64), colind, rowptr), shape=shape)
    else:
        rng = np.random.default_rng(8)
        S = sp.random(m, n, density=0.3, random_state=9, format="csr")
        S.data = rng.standard_normal(S.nnz)
    nsv = 6
    v0 = P.start_vector(min(m, n), 1)
    r = oracle_mod.svd_cross(S.indptr, S.indices, S.data, shape, v0, nsv, 30, tol=1e-12, largest=largest)
    d = np.linalg.svd(S.toarray(), compute_uv=False)
    d = d if largest else d[::-1]
    assert r.nconv >= nsv and r.reason == 1
    np.testing.assert_allclose(r.sigma[:nsv], d[:nsv], rtol=1e-12)
    assert r.U.shape == (m, r.nconv) and r.V.shape == (n, r.nconv)
    assert np.abs(r.U.T @ r.U - np.eye(r.nconv)).max() < 1e-13
    for i in range(nsv):
        res = np.hypot(np.linalg.norm(S @ r.V[:, i] - r.sigma[i] * r.U[:, i]),
                       np.linalg.norm(S.T @ r.U[:, i] - r.sigma[i] * r.V[:, i])) / (r.sigma[i] * np.sqrt(2))
        assert res == pytest.approx(r.rel_error[i], rel=1e-6, abs=1e-15)
        assert res < 1e-10


def test_create_aij_rejects_bad_arguments():
    import slepc_b200 as S

    L = S.lib()
    h = ctypes.c_void_p()
    rowptr = np.array([0, 2, 3], dtype=np.int32)
    vals = np.ones(3, dtype=np.float32)
    bad_col = np.array([0, 5, 1], dtype=np.int32)
    assert L.b200_mat_create_aij(2, 4, 3, S._i(rowptr), S._i(bad_col), vals.ctypes.data, S.SCALAR_F32, None,
                                 ctypes.byref(h)) == 1
    cols = np.array([0, 3, 1], dtype=np.int32)
    assert L.b200_mat_create_aij(2, 4, 4, S._i(rowptr), S._i(cols), vals.ctypes.data, S.SCALAR_F32, None,
                                 ctypes.byref(h)) == 1
    assert L.b200_mat_create_aij(2, 4, 3, S._i(rowptr), S._i(cols), vals.ctypes.data, 7, None,
                                 ctypes.byref(h)) == 1
    assert "scalar type" in L.b200_last_error().decode()
    assert L.b200_svd_set_dimensions(None, 0, 0, 0) == 1
    assert L.b200_svd_set_which_singular_triplets(None, 5) == 1
