"""GPU parity of the SVD cross path against the CPU oracle and dense LAPACK.

Covers the general AIJ matrix (FP32 and FP64 value storage) with its explicit
transpose, the warp-tile SpMV with long-row segments (the power-law columns of
A make rows of A^T with thousands of nonzeros), the A^T A shell of
MatMult_Cross, and the b200_svd_* solver (SVDCROSS).  Every call goes through
the C ABI.

Tolerances: rows of at most 256 nonzeros are summed in index order and match
the oracle bit for bit; a longer row is summed as fixed-order segment partials,
so it is compared within 1e-12 of the sum of |products| (a bound on the
rounding of either order).  Singular values agree with the oracle to 1e-10
relative, singular subspaces to a sine of 1e-8.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from slepc_b200 import problems as P
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _dev(a):
    return _torch().from_numpy(np.ascontiguousarray(a)).cuda()


def _nan(n):
    torch = _torch()
    return torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")


def _scipy(csr, shape):
    return sp.csr_matrix((np.asarray(csr[2], dtype=np.float64), csr[1], csr[0]), shape=shape)


def _mat(b200, csr, shape, dtype):
    return b200.Mat().createAIJ((csr[0], csr[1], np.asarray(csr[2]).astype(dtype)), size=shape, dtype=dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_aij_mult_and_transpose_vs_oracle(b200, oracle_mod, dtype):
    torch = _torch()
    m, n = 9000, 1200
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=3)
    S = _scipy(csr, (m, n))
    rt, ct, vt = oracle_mod.csr_transpose(csr[0], csr[1], S.data, (m, n))
    T = sp.csr_matrix((vt, ct, rt), shape=(n, m))
    lens = np.diff(rt)
    assert lens.max() > 2 * 4096, "the transpose must have rows of several segments"
    A = _mat(b200, csr, (m, n), dtype)
    assert A.getSizes() == (m, n)
    rng = np.random.default_rng(0)
    x, z = rng.standard_normal(n), rng.standard_normal(m)
    xd, zd, y, yt = _dev(x), _dev(z), _nan(m), _nan(n)
    A.mult(xd.data_ptr(), y.data_ptr())
    A.multTranspose(zd.data_ptr(), yt.data_ptr())
    torch.cuda.synchronize()
    y, yt = y.cpu().numpy(), yt.cpu().numpy()
    assert np.array_equal(y, oracle_mod.spmv(S, x))
    ref = oracle_mod.spmv(T, z)
    short = lens <= 256
    assert short.any() and (~short).any()
    assert np.array_equal(yt[short], ref[short])
    bound = 1e-12 * (abs(T) @ np.abs(z))
    assert np.all(np.abs(yt - ref) <= bound)
    # deterministic: a second product gives the same bits
    yt2 = _nan(n)
    A.multTranspose(zd.data_ptr(), yt2.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(yt2.cpu().numpy(), yt)
    assert A.norm() == pytest.approx(np.abs(S).sum(axis=1).max(), rel=1e-12)


def test_cross_shell_vs_oracle(b200, oracle_mod):
    torch = _torch()
    m, n = 6000, 900
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=4)
    S = _scipy(csr, (m, n))
    A = _mat(b200, csr, (m, n), np.float32)
    C = b200.Mat().createCross(A)
    assert C.getSizes() == (n, n)
    x = np.random.default_rng(1).standard_normal(n)
    y = _nan(n)
    C.mult(_dev(x).data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    w = oracle_mod.spmv(S, x)
    rt, ct, vt = oracle_mod.csr_transpose(csr[0], csr[1], S.data, (m, n))
    T = sp.csr_matrix((vt, ct, rt), shape=(n, m))
    ref = oracle_mod.spmv(T, w)
    assert np.all(np.abs(y.cpu().numpy() - ref) <= 1e-12 * (abs(T) @ np.abs(w)))


def _gpu_svd(b200, A, v0, nsv, ncv, tol, which=0):
    E = b200.SVD().create()
    E.setOperators(A)
    E.setDimensions(nsv, ncv)
    E.setTolerances(tol)
    E.setWhichSingularTriplets(which)
    E.setInitialSpace(v0)
    E.solve()
    k = E.getConverged()
    trip = [E.getSingularTriplet(i) for i in range(k)]
    sig = np.array([t[0] for t in trip])
    U = np.array([t[1] for t in trip]).T
    V = np.array([t[2] for t in trip]).T
    err = np.array([E.computeError(i) for i in range(k)])
    return E, sig, U, V, err


def _check_vs_oracle(sig, U, V, err, ref, nsv, tol_err):
    k = min(len(sig), ref.nconv)
    assert k >= nsv
    assert np.all(np.diff(sig) <= 0), "largest singular values come first"
    np.testing.assert_allclose(sig[:k], ref.sigma[:k], rtol=1e-10)
    assert err.max() <= tol_err and ref.rel_error.max() <= tol_err
    assert np.abs(U.T @ U - np.eye(U.shape[1])).max() <= 1e-12
    for lam, s in H.eigenspace_sines(sig[:nsv], V[:, :nsv], ref.sigma[:k], ref.V[:, :k], rtol=1e-8):
        assert s <= 1e-8, (lam, s)
    for lam, s in H.eigenspace_sines(sig[:nsv], U[:, :nsv], ref.sigma[:k], ref.U[:, :k], rtol=1e-8):
        assert s <= 1e-8, (lam, s)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_svd_largest_vs_oracle_and_dense(b200, oracle_mod, dtype):
    m, n, nsv, ncv, tol = 4000, 700, 10, 30, 1e-12
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=5)
    S = _scipy(csr, (m, n))
    v0 = P.start_vector(n, 1)
    A = _mat(b200, csr, (m, n), dtype)
    E, sig, U, V, err = _gpu_svd(b200, A, v0, nsv, ncv, tol)
    ref = oracle_mod.svd_cross(csr[0], csr[1], S.data, (m, n), v0, nsv, ncv, tol=tol)
    assert E.getConvergedReason() == 1 and E.getIterationNumber() == ref.its
    _check_vs_oracle(sig, U, V, err, ref, nsv, 1e-10)
    dense = np.linalg.svd(S.toarray(), compute_uv=False)
    np.testing.assert_allclose(sig[:nsv], dense[:nsv], rtol=1e-10)


def test_svd_fp32_and_fp64_storage_agree_bitwise(b200):
    """Values representable in float32: FP32 storage widens them exactly, so both
    storages give the same bits."""
    m, n = 3000, 500
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=6)
    v0 = P.start_vector(n, 2)
    out = []
    for dt in (np.float32, np.float64):
        A = _mat(b200, csr, (m, n), dt)
        out.append(_gpu_svd(b200, A, v0, 6, 24, 1e-10)[1:])
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_svd_fewer_rows_than_columns(b200, oracle_mod):
    """m < n: the operator is A A^T and u, v exchange roles (SVDSetUp's swap)."""
    m, n, nsv, ncv, tol = 500, 2500, 8, 24, 1e-12
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=7)
    S = _scipy(csr, (m, n))
    v0 = P.start_vector(m, 3)
    A = _mat(b200, csr, (m, n), np.float32)
    E, sig, U, V, err = _gpu_svd(b200, A, v0, nsv, ncv, tol)
    assert U.shape[0] == m and V.shape[0] == n
    ref = oracle_mod.svd_cross(csr[0], csr[1], S.data, (m, n), v0, nsv, ncv, tol=tol)
    _check_vs_oracle(sig, U, V, err, ref, nsv, 1e-10)
    # A v = sigma u directly
    r = S @ V[:, 0] - sig[0] * U[:, 0]
    assert np.linalg.norm(r) <= 1e-9 * sig[0]


def test_svd_smallest_full_rank(b200):
    rng = np.random.default_rng(8)
    m, n = 600, 80
    D = sp.random(m, n, density=0.3, random_state=9, format="csr")
    D.data = rng.standard_normal(D.nnz)
    csr = (D.indptr.astype(np.int32), D.indices.astype(np.int32), D.data)
    A = _mat(b200, csr, (m, n), np.float64)
    E, sig, U, V, err = _gpu_svd(b200, A, P.start_vector(n, 4), 4, 40, 1e-10, which=1)
    dense = np.linalg.svd(D.toarray(), compute_uv=False)[::-1]
    assert len(sig) >= 4 and np.all(np.diff(sig) >= 0)
    np.testing.assert_allclose(sig[:4], dense[:4], rtol=1e-8)
    assert err[:4].max() <= 1e-8


def test_svd_solve_aij_host_matches_objects(b200):
    m, n = 2500, 400
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=10)
    v0 = P.start_vector(n, 5)
    A = _mat(b200, csr, (m, n), np.float32)
    _, sig, U, V, err = _gpu_svd(b200, A, v0, 6, 20, 1e-10)
    r = b200.svd_solve_aij_host(csr, (m, n), v0, 6, 20, tol=1e-10, dtype=np.float32)
    assert r["nconv"] == len(sig)
    assert np.array_equal(r["sigma"], sig) and np.array_equal(r["U"], U) and np.array_equal(r["V"], V)
    np.testing.assert_array_equal(r["rel_error"], err)


def test_svd_call_order_and_argument_errors(b200):
    m, n = 300, 100
    csr = P.powerlaw_rect(m, n, 10, 1.8, seed=11)
    A = _mat(b200, csr, (m, n), np.float32)
    E = b200.SVD().create()
    E.setOperators(A)
    with pytest.raises(b200.B200Error) as e:
        E.getSingularTriplet(0)
    assert e.value.status == 7
    with pytest.raises(b200.B200Error):
        A.setSpMVSchedule(b200.Mat.ROWBLOCK)
    Q = b200.Mat().createAIJ(P.laplacian_2d(8))
    with pytest.raises(b200.B200Error):
        b200.Mat().createCross(Q)
    with pytest.raises(b200.B200Error):
        Q.multTranspose(0, 0)
    C = b200.Mat().createCross(A)
    Eps = b200.EPS().create()
    Eps.setOperators(C)  # square: accepted
    with pytest.raises(b200.B200Error):
        Eps.setOperators(A)  # rectangular: rejected


def test_svd_cross_full_size_properties(b200):
    """The 2,000,000 x 500,000 power-law matrix (20 nonzeros per row, FP32
    values): the 32 largest triplets at tol 1e-7 with ncv 96, every relative
    error below the tolerance, singular values descending, U orthonormal."""
    m, n, nsv, ncv, tol = 2_000_000, 500_000, 32, 96, 1e-7
    csr = P.powerlaw_rect(m, n, 20, 1.8, seed=0)
    A = _mat(b200, csr, (m, n), np.float32)
    E = b200.SVD().create()
    E.setOperators(A)
    E.setDimensions(nsv, ncv)
    E.setTolerances(tol)
    E.setInitialSpace(P.start_vector(n, 0))
    E.solve()
    k = E.getConverged()
    assert E.getConvergedReason() == 1 and k >= nsv
    sig = np.array([E.getValue(i) for i in range(k)])
    assert np.all(np.diff(sig) <= 0)
    err = np.array([E.computeError(i) for i in range(nsv)])
    assert err.max() <= tol, err.max()
    U = np.array([E.getSingularTriplet(i)[1] for i in range(4)]).T
    assert np.abs(U.T @ U - np.eye(4)).max() <= 1e-12
    u_ptr, v_ptr = E.getVectorPointers(0)
    assert u_ptr and v_ptr
