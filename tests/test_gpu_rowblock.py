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
