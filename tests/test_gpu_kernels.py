"""GPU parity of the individual kernels against the CPU oracle and SLEPc's golden outputs.

Every call goes through the C ABI (libslepc_b200.so).  Tolerances: the
integer-valued BV fixtures of SLEPc's tests are exact in FP64 and are
compared bit for bit; floating-point results of longer sums (different
summation order than BLAS) are compared to 1e-13 relative.
"""
import numpy as np
import pytest

from slepc_b200 import problems as P
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _random_csr(n, rng, max_row=70, empty_every=17):
    """Ragged CSR with empty rows, short rows and a few long rows (symmetric not required)."""
    lens = rng.integers(0, 9, size=n)
    lens[::empty_every] = 0
    lens[rng.integers(0, n, size=max(1, n // 200))] = max_row
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(lens, out=rowptr[1:])
    colind = np.concatenate([np.sort(rng.choice(n, size=l, replace=False)) for l in lens]).astype(np.int32)
    vals = rng.standard_normal(rowptr[-1])
    return rowptr, colind, vals


@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_spmv_all_lane_widths_vs_oracle(b200, oracle_mod, lanes):
    torch = _torch()
    rng = np.random.default_rng(lanes)
    n = 5003
    csr = _random_csr(n, rng)
    x = rng.standard_normal(n)
    ref = oracle_mod.spmv(P.to_scipy(csr), x)
    d = [torch.from_numpy(np.asarray(a)).cuda() for a in csr]
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    b200._check(b200.lib().b200_csr_spmv(n, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), xd.data_ptr(),
                                         yd.data_ptr(), lanes, None))
    torch.cuda.synchronize()
    np.testing.assert_allclose(yd.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("schedule", [0, 1, 2, 3])
def test_spmv_laplacian_via_mat_bit_exact(b200, oracle_mod, schedule):
    """Mat SpMV (row blocks / warp tiles): rows summed in index order, so it matches the
    oracle's sequential row loop bit for bit."""
    torch = _torch()
    csr = P.laplacian_3d(40, 33, 29)
    n = len(csr[0]) - 1
    A = b200.Mat().createAIJ(csr)
    A.setSpMVSchedule(schedule)
    assert A.getLanes() == 8
    x = P.start_vector(n, 4)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    A.mult(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(yd.cpu().numpy(), oracle_mod.spmv(P.to_scipy(csr), x))


@pytest.mark.parametrize("schedule", [0, 1, 2, 3])
def test_spmv_mat_ragged_long_rows(b200, oracle_mod, schedule):
    """Empty rows, short rows, and rows longer than a tile (4096 / 256 nonzeros)."""
    torch = _torch()
    rng = np.random.default_rng(3)
    n = 20011
    lens = rng.integers(0, 12, size=n)
    lens[::13] = 0
    lens[[5, 777, 20010]] = [5000, 9000, 4097]
    lens[[100, 101, 102, 9000, 9031]] = [40, 200, 33, 256, 32]  # tile rows beside sliced-ELL rows
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rowptr[1:])
    colind = np.concatenate([np.sort(rng.choice(n, size=l, replace=False)) for l in lens]).astype(np.int32)
    vals = rng.standard_normal(int(rowptr[-1]))
    csr = (rowptr.astype(np.int32), colind, vals)
    A = b200.Mat().createAIJ(csr)
    A.setSpMVSchedule(schedule)
    x = rng.standard_normal(n)
    xd = torch.from_numpy(x).cuda()
    yd = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    A.mult(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    ref = oracle_mod.spmv(P.to_scipy(csr), x)
    y = yd.cpu().numpy()
    short = lens <= (4096 if schedule == 0 else 256)
    np.testing.assert_array_equal(y[short], ref[short])
    np.testing.assert_allclose(y[~short], ref[~short], rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("case", ["laplacian", "ragged"])
def test_bv_mat_mult_block_vs_columns(b200, oracle_mod, case):
    """BVMatMult (block SpMV over the active columns) against the oracle's SpMV column by column:
    bit for bit on rows the sliced-ELL slices hold (index-order sums, products and sums rounded
    separately), to 1e-12 relative on the rows longer than a slice."""
    rng = np.random.default_rng(7)
    if case == "laplacian":
        csr = P.laplacian_3d(30, 27, 25)
        n = len(csr[0]) - 1
        lens = np.diff(csr[0])
    else:
        n = 9001
        lens = rng.integers(0, 12, size=n)
        lens[::11] = 0
        lens[[3, 4000, 9000]] = [700, 33, 64]
        rowptr = np.zeros(n + 1, dtype=np.int32)
        np.cumsum(lens, out=rowptr[1:])
        colind = np.concatenate([np.sort(rng.choice(n, size=l, replace=False)) for l in lens]).astype(np.int32)
        csr = (rowptr, colind, rng.standard_normal(int(rowptr[-1])))
    A = b200.Mat().createAIJ(csr)
    m = 21
    X = rng.standard_normal((n, m))
    V = b200.BV().create(n, m)
    Y = b200.BV().create(n, m + 1)
    V.setColumns(X)
    for lk in ((0, m), (2, 19)):
        V.setActiveColumns(*lk)
        Y.setActiveColumns(1, 1 + lk[1] - lk[0])
        V.matMult(A, Y)
        got = Y.getColumns()
        As = P.to_scipy(csr)
        short = lens <= 32
        for j in range(lk[1] - lk[0]):
            ref = oracle_mod.spmv(As, X[:, lk[0] + j])
            y = got[:, 1 + j]
            np.testing.assert_array_equal(y[short], ref[short])
            np.testing.assert_allclose(y[~short], ref[~short], rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    V.destroy()
    Y.destroy()
    A.destroy()


def test_bv_test1_golden_ops(b200):
    """src/sys/classes/bv/tests/test1.c: BVMult, BVMultVec, BVDot, BVDotVec, BVMultInPlace, BVScale, BVNorm."""
    torch = _torch()
    g = H.golden("bv_test1.json")
    X0, Y0, Q = H.bv_test1_fixture()
    n, k, l = g["n"], g["k"], g["l"]
    X = b200.BV().create(n, k)
    Y = b200.BV().create(n, l)
    X.setColumns(X0)
    Y.setColumns(Y0)
    Y.mult(2.0, 1.0, X, Q)
    np.testing.assert_array_equal(Y.getColumns().T, np.array(g["Y_after_mult"]))
    z = np.zeros(k)
    z[0] = 2.0
    for i in range(1, k):
        z[i] = -0.5 * z[i - 1]
    y0 = torch.from_numpy(Y.getColumn(0)).cuda()
    X.multVec(-1.0, 1.0, y0.data_ptr(), z)
    Y.setColumn(0, y0.cpu().numpy())
    np.testing.assert_array_equal(Y.getColumns().T, np.array(g["Y_after_multvec"]))
    M = X.dot(Y)
    np.testing.assert_array_equal(M, np.array(g["M_after_dot"]))
    q = X.dotVec(torch.from_numpy(Y.getColumn(0)).cuda().data_ptr(), k)
    np.testing.assert_array_equal(q, np.array(g["z_after_dotvec"]))
    X.multInPlace(Q, 1, l)
    X.scale(2.0)
    np.testing.assert_array_equal(X.getColumns().T, np.array(g["X_after_multinplace_scale2"]))
    assert float("%g" % X.normColumn(0)) == g["norm2_X0"]
    assert float("%g" % X.norm()) == g["norm_fro"]


def test_bv_test2_golden_orthogonalization(b200):
    """src/sys/classes/bv/tests/test2.c: BVOrthogonalizeColumn, BVOrthogonalize (with R), BVOrthogonalizeVec."""
    torch = _torch()
    g = H.golden("bv_test2.json")
    n, k = g["n"], g["k"]
    X0 = H.bv_test2_fixture(n, k)
    eps = np.finfo(float).eps
    X = b200.BV().create(n, k)
    X.setColumns(X0)
    for j in range(k):
        _, nrm, _ = X.orthogonalizeColumn(j)
        X.scaleColumn(j, 1.0 / nrm)
    Xh = X.getColumns()
    assert np.abs(Xh.T @ Xh - np.eye(k)).sum(axis=0).max() < 100 * eps
    Y = b200.BV().create(n, k)
    Y.setColumns(X0)
    R = Y.orthogonalize(k)
    Yh = Y.getColumns()
    assert np.abs(Yh.T @ Yh - np.eye(k)).sum(axis=0).max() < 100 * eps
    assert np.linalg.norm(X0 - Yh @ R) < 100 * eps
    e = torch.ones(n, dtype=torch.float64, device="cuda")
    _, nrm, _ = X.orthogonalizeVec(e.data_ptr(), k)
    assert float("%.5f" % nrm) == g["norm_ones_after_orth"]


@pytest.mark.parametrize("n,m,j", [(7, 4, 3), (1000, 20, 0), (1000, 20, 1), (4099, 41, 40), (200003, 81, 60),
                                   (65536, 97, 96)])
def test_orthogonalize_column_vs_oracle(b200, oracle_mod, n, m, j):
    """Random orthonormal basis plus a vector with large components on it (forces the DGKS refinement)."""
    rng = np.random.default_rng(n + j)
    Q, _ = np.linalg.qr(rng.standard_normal((n, max(j, 1))))
    V = np.zeros((n, m), order="F")
    V[:, :j] = Q[:, :j]
    V[:, j] = (Q[:, :j] @ (10 * rng.standard_normal(j)) if j else 0) + 1e-2 * rng.standard_normal(n)
    Vo = V.copy(order="F")
    Ho, no, lo = oracle_mod.bv_orthogonalize_column(Vo, j, normalize=False)
    bv = b200.BV().create(n, m)
    bv.setColumns(V[:, : j + 1])
    Hg, ng, lg = bv.orthogonalizeColumn(j)
    assert lg == lo
    np.testing.assert_allclose(ng, no, rtol=1e-12)
    np.testing.assert_allclose(Hg, Ho, rtol=1e-11, atol=1e-13 * np.abs(Ho).max())
    np.testing.assert_allclose(bv.getColumn(j), Vo[:, j], rtol=0, atol=1e-12 * np.abs(Vo[:, j]).max())


def test_orthonormalize_zero_and_dependent_columns(b200, oracle_mod):
    n = 3000
    rng = np.random.default_rng(9)
    Q, _ = np.linalg.qr(rng.standard_normal((n, 5)))
    V = np.zeros((n, 8), order="F")
    V[:, :5] = Q
    V[:, 5] = Q @ np.arange(1.0, 6.0)  # exactly in the span: linearly dependent
    bv = b200.BV().create(n, 8)
    bv.setColumns(V[:, :7])
    nrm, lindep = bv.orthonormalizeColumn(5)
    Vo = V.copy(order="F")
    _, no, lo = oracle_mod.bv_orthogonalize_column(Vo, 5, normalize=True)
    # SLEPc's DGKS test (bvorthog.c:176-187) sees the rounding residue of an exactly dependent vector as a
    # new direction: the norm collapses by ~1e-16 but the flag follows the reference
    assert lindep == lo
    assert nrm < 1e-12 * np.linalg.norm(V[:, 5]) and no < 1e-12 * np.linalg.norm(V[:, 5])
    # zero column: norm exactly zero, flagged dependent, left unscaled
    nrm0, lindep0 = bv.orthonormalizeColumn(6)
    assert nrm0 == 0.0 and lindep0
    assert np.all(bv.getColumn(6) == 0.0)


@pytest.mark.parametrize("n,nv,s,e,nconv", [(10, 5, 1, 3, 0), (1000, 32, 3, 20, 3), (100003, 80, 10, 66, 10),
                                            (4097, 97, 0, 97, 0), (77, 40, 39, 40, 0)])
def test_multinplace_vs_oracle(b200, oracle_mod, n, nv, s, e, nconv):
    rng = np.random.default_rng(n)
    V = np.asfortranarray(rng.standard_normal((n, nv + 1)))
    Q = np.asfortranarray(rng.standard_normal((nv + 1, nv + 1)))
    Vo = V.copy(order="F")
    oracle_mod.bv_multinplace(Vo, nconv, nv, Q, s, e)
    bv = b200.BV().create(n, nv + 1)
    bv.setColumns(V)
    bv.setActiveColumns(nconv, nv)
    bv.multInPlace(Q, s, e)
    G = bv.getColumns()
    np.testing.assert_allclose(G, Vo, rtol=1e-12, atol=1e-12 * np.abs(Vo).max())


def test_mat_lanczos_vs_oracle_three_term(b200, oracle_mod):
    """BVMatLanczos on a 2-D Laplacian: T entries equal the oracle's restated Lanczos to 1e-10."""
    csr = P.laplacian_2d(60, 61)
    n = len(csr[0]) - 1
    A = b200.Mat().createAIJ(csr)
    v0 = P.start_vector(n, 2)
    v0 /= np.linalg.norm(v0)
    bv = b200.BV().create(n, 31)
    bv.setColumn(0, v0)
    alpha, beta_v, m, beta, bd = bv.matLanczos(A, 0, 30)
    assert m == 30 and not bd
    # reference: same recurrence on the CPU with full reorthogonalisation (oracle building blocks)
    Vo = np.zeros((n, 31), order="F")
    Vo[:, 0] = v0
    As = P.to_scipy(csr)
    ao, bo = np.zeros(30), np.zeros(30)
    for j in range(30):
        Vo[:, j + 1] = oracle_mod.spmv(As, Vo[:, j])
        Hj, nrm, _ = oracle_mod.bv_orthogonalize_column(Vo, j + 1, normalize=True)
        ao[j], bo[j] = Hj[j], nrm
    np.testing.assert_allclose(alpha[:30], ao, rtol=1e-10)
    np.testing.assert_allclose(beta_v[:30], bo, rtol=1e-8)
    Vg = bv.getColumns(31)
    assert np.abs(Vg.T @ Vg - np.eye(31)).max() < 1e-13


@pytest.mark.parametrize("nx,ny", [(48, 16), (7, 33), (250, 120)])
def test_bv_mult_alpha_beta_vs_numpy(b200, nx, ny):
    """BVMult Y = alpha X Q + beta Y: the row-panel tensor-core product and the column kernel it
    falls back to when X's panel and Q do not fit shared memory (250 x 120) against numpy in FP64."""
    rng = np.random.default_rng(nx * 1000 + ny)
    n = 20011
    X0 = rng.standard_normal((n, nx))
    Y0 = rng.standard_normal((n, ny))
    Q = rng.standard_normal((nx, ny))
    X = b200.BV().create(n, nx)
    Y = b200.BV().create(n, ny)
    X.setColumns(X0)
    Y.setColumns(Y0)
    Y.mult(-0.7, 1.3, X, Q)
    ref = -0.7 * X0 @ Q + 1.3 * Y0
    got = Y.getColumns()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(X0).max() * np.abs(Q).max() * nx
    Y.setColumns(Y0)
    Y.mult(1.0, 0.0, X, Q)
    assert np.abs(Y.getColumns() - X0 @ Q).max() <= 1e-13 * np.abs(X0).max() * np.abs(Q).max() * nx
    X.destroy()
    Y.destroy()


@pytest.mark.parametrize("nx,ny", [(16, 16), (20, 9), (48, 48), (33, 40), (64, 64), (130, 70)])
def test_bv_dot_gram_tiles_vs_numpy(b200, nx, ny):
    """BVDot M = Y^T X through every Gram tile width (16, 32, 48, 64 columns, several tiles per
    side) and both row-block counts against numpy in FP64."""
    rng = np.random.default_rng(nx * 7 + ny)
    n = 50021
    X0 = rng.standard_normal((n, nx))
    Y0 = rng.standard_normal((n, ny))
    X = b200.BV().create(n, nx)
    Y = b200.BV().create(n, ny)
    X.setColumns(X0)
    Y.setColumns(Y0)
    M = X.dot(Y)
    ref = Y0.T @ X0
    assert M.shape == ref.shape
    assert np.abs(M - ref).max() <= 1e-13 * n
    np.testing.assert_array_equal(M, X.dot(Y))  # deterministic
    X.destroy()
    Y.destroy()
