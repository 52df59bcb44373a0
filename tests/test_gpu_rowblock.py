"""Row-major block kernels of the mixed form against numpy FP64 references.

The tensor-core Gram product (tcgen05 kind::tf32) reads its FP32 inputs with 10
mantissa bits, so it is checked elementwise against the FP64 product within a
TF32 bound, 1.25 * 2^-9 * (|X|^T |Y|) (each input rounded by less than 2^-10
relative, plus FP32 accumulation); the FP64 Gram (FP64 MMAs for 64 columns) is checked to 1e-12.  Sizes
include a partial last tile (n not a multiple of the tile height), a block
narrower than one tile, both block widths (64, 128), X^T X and X^T Y.
"""
import numpy as np
import pytest

import slepc_b200 as S

pytestmark = pytest.mark.gpu


def _blocks(n, bp, seed, scale_cols=False):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, bp)).astype(np.float32)
    Y = rng.standard_normal((n, bp)).astype(np.float32)
    if scale_cols:
        X *= np.geomspace(1.0, 1e-3, bp).astype(np.float32)
    return X, Y


def _gram(X, Y, tc):
    import torch

    n, bp = X.shape
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    Yd = torch.from_numpy(np.ascontiguousarray(Y)).cuda() if Y is not None else None
    Gd = torch.full((bp, bp), np.nan, dtype=torch.float64, device="cuda")
    S.rowblock_gram(n, bp, Xd.data_ptr(), Yd.data_ptr() if Yd is not None else None, tc, Gd.data_ptr())
    torch.cuda.synchronize()
    return Gd.cpu().numpy()


@pytest.mark.parametrize("n,bp", [(10007, 64), (100, 64), (300001, 64), (5003, 128), (262147, 128)])
@pytest.mark.parametrize("cross", [False, True])
def test_tensor_core_gram_within_tf32_bound(n, bp, cross):
    X, Y = _blocks(n, bp, n + bp, scale_cols=True)
    Yr = Y if cross else X
    ref = X.astype(np.float64).T @ Yr.astype(np.float64)
    bound = np.abs(X.astype(np.float64)).T @ np.abs(Yr.astype(np.float64))
    G = _gram(X, Y if cross else None, True)
    assert np.isfinite(G).all()
    err = np.abs(G - ref)
    # TF32 inputs (relative error < 2^-10 each) plus FP32 accumulation within a CTA
    assert (err <= 1.25 * 2.0 ** -9 * bound + 1e-30).all(), (err / bound).max()
    # the truncation error is mostly a common scale: after it the product is far closer than the bound
    s = np.trace(G) / np.trace(ref) if not cross else 1.0
    if not cross:
        assert np.abs(G / s - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("n,bp", [(10007, 64), (5003, 128), (262147, 64), (31, 64)])
def test_fp64_gram_exact_products(n, bp):
    X, Y = _blocks(n, bp, 7)
    ref = X.astype(np.float64).T @ Y.astype(np.float64)
    G = _gram(X, Y, False)
    np.testing.assert_allclose(G, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_gram_deterministic():
    X, Y = _blocks(77777, 64, 3)
    assert np.array_equal(_gram(X, None, True), _gram(X, None, True))
    assert np.array_equal(_gram(X, Y, False), _gram(X, Y, False))


def test_gram_rejects_bad_width():
    import torch

    # real buffers: only the argument check may run
    Xd = torch.zeros((100, 96), dtype=torch.float32, device="cuda")
    Gd = torch.zeros((96, 96), dtype=torch.float64, device="cuda")
    with pytest.raises(S.B200Error):
        S.rowblock_gram(100, 96, Xd.data_ptr(), None, True, Gd.data_ptr())


def _irregular_csr(n, seed):
    # rows of 0..9 nonzeros plus a few rows longer than a 32-row slice admits (the rest path)
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 10, n)
    lens[rng.choice(n, 7, replace=False)] = rng.integers(40, 90, 7)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    colind = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens]).astype(np.int32)
    vals = rng.standard_normal(int(rowptr[-1]))
    return rowptr, colind, vals


@pytest.mark.parametrize("bp", [64, 128])
@pytest.mark.parametrize("x32", [True, False])
def test_block_spmv_filter_step_against_numpy(bp, x32):
    # Y = alpha (A X - shift X) - beta Z, the Chebyshev filter step, against an FP64 reference on the
    # same (FP32-rounded when x32) values: FP32 products within 2^-20 of |A||X|, FP64 within 1e-13
    import scipy.sparse as sp
    import torch

    n = 5003
    rowptr, colind, vals = _irregular_csr(n, bp + int(x32))
    A = S.Mat().createAIJ((rowptr, colind, vals))
    dt = np.float32 if x32 else np.float64
    rng = np.random.default_rng(5)
    X = rng.standard_normal((n, bp)).astype(dt)
    Z = rng.standard_normal((n, bp)).astype(dt)
    Xd, Zd = torch.from_numpy(X).cuda(), torch.from_numpy(Z).cuda()
    Yd = torch.full((n, bp), np.nan, dtype=Xd.dtype, device="cuda")
    alpha, shift, beta = 0.7, 0.3, 0.2
    S.rowblock_spmm(A, bp, Xd.data_ptr(), Yd.data_ptr(), Zd.data_ptr(), alpha, shift, beta, x32=x32)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy().astype(np.float64)
    v = vals.astype(np.float32).astype(np.float64) if x32 else vals
    M = sp.csr_matrix((v, colind, rowptr), shape=(n, n))
    X64, Z64 = X.astype(np.float64), Z.astype(np.float64)
    ref = alpha * (M @ X64 - shift * X64) - beta * Z64
    bound = alpha * (abs(M) @ np.abs(X64) + shift * np.abs(X64)) + beta * np.abs(Z64)
    tol = 2.0 ** -20 if x32 else 1e-13
    assert np.isfinite(Y).all()
    assert (np.abs(Y - ref) <= tol * bound + 1e-300).all(), (np.abs(Y - ref) / np.maximum(bound, 1e-300)).max()
    A.destroy()
