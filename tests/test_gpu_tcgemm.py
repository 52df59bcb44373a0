"""Tensor-core FP32 GEMM of the neural operator (b200_tc_sgemm) against numpy FP64 products.

The kernel splits every FP32 input into a TF32 high part and the remainder and
sums three tcgen05 TF32 products (hi*hi + hi*lo + lo*hi) in the FP32 TMEM
accumulator, so it must be as accurate as an FP32 GEMM: each element within
4e-6 of |A||B| (elementwise products of absolute values), a bound plain TF32
(about 2^-10 per input) misses by two orders of magnitude.  Cases cover both
orientations (m >= n and the transposed path m < n), column-major and strided
views (the transposed operands of the backward pass), batches with beta,
partial tiles, the split-depth path with its ordered reduction, the sum over
the batch (weight gradients), an empty depth, and bit-identical repeats.
"""
import numpy as np
import pytest

import slepc_b200 as S

pytestmark = pytest.mark.gpu

TOL = 4e-6


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _run(A, B, C0, alpha, beta, Aview, Bview, Cview, batch, m, n, k, split=False, sum_batch=False):
    import torch

    Ad, Bd, Cd = _dev(A), _dev(B), _dev(C0)
    S.tc_sgemm(batch, m, n, k, alpha, (Ad.data_ptr(), *Aview), (Bd.data_ptr(), *Bview), beta,
               (Cd.data_ptr(), *Cview), split=split, sum_batch=sum_batch)
    torch.cuda.synchronize()
    return Cd.cpu().numpy()


def _check(C, ref, bound):
    err = np.abs(C.astype(np.float64) - ref)
    assert np.isfinite(C).all()
    assert (err <= TOL * bound + 1e-30).all(), (err / np.maximum(bound, 1e-300)).max()


@pytest.mark.parametrize("m,n,k", [(300, 50, 70), (20, 500, 33), (129, 17, 1), (1000, 64, 300), (64, 1000, 4096)])
def test_row_major(m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    A = rng.standard_normal((m, k)).astype(np.float32)
    B = rng.standard_normal((k, n)).astype(np.float32)
    C = _run(A, B, np.full((m, n), np.nan, np.float32), 1.0, 0.0, (k, 1, 0), (n, 1, 0), (n, 1, 0), 1, m, n, k)
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    _check(C, A64 @ B64, np.abs(A64) @ np.abs(B64))


def test_transposed_views_and_beta():
    rng = np.random.default_rng(3)
    m, n, k = 200, 40, 96
    At = rng.standard_normal((k, m)).astype(np.float32)   # A = At^T: element (i, kk) at kk*m + i
    Bt = rng.standard_normal((n, k)).astype(np.float32)   # B = Bt^T: element (kk, j) at j*k + kk
    C0 = rng.standard_normal((n, m)).astype(np.float32)   # C stored transposed: element (i, j) at j*m + i
    C = _run(At, Bt, C0, 0.5, -2.0, (1, m, 0), (1, k, 0), (1, m, 0), 1, m, n, k)
    A64, B64 = At.T.astype(np.float64), Bt.T.astype(np.float64)
    ref = 0.5 * A64 @ B64 - 2.0 * C0.T.astype(np.float64)
    bound = 0.5 * np.abs(A64) @ np.abs(B64) + 2.0 * np.abs(C0.T)
    _check(C.T, ref, bound)


def test_batched_strided():
    rng = np.random.default_rng(5)
    batch, m, n, k = 7, 90, 33, 50
    A = rng.standard_normal((batch, m, k)).astype(np.float32)
    B = rng.standard_normal((batch, k, n)).astype(np.float32)
    C0 = rng.standard_normal((batch, m, n)).astype(np.float32)
    C = _run(A, B, C0, 1.0, 1.0, (k, 1, m * k), (n, 1, k * n), (n, 1, m * n), batch, m, n, k)
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    ref = A64 @ B64 + C0
    bound = np.abs(A64) @ np.abs(B64) + np.abs(C0)
    _check(C, ref, bound)


@pytest.mark.parametrize("k", [100000, 4099])
def test_split_depth(k):
    rng = np.random.default_rng(k)
    m, n = 32, 24
    A = rng.standard_normal((m, k)).astype(np.float32)
    B = rng.standard_normal((k, n)).astype(np.float32)
    C = _run(A, B, np.zeros((m, n), np.float32), 1.0, 0.0, (k, 1, 0), (n, 1, 0), (n, 1, 0), 1, m, n, k, split=True)
    A64, B64 = A.astype(np.float64), B.astype(np.float64)
    _check(C, A64 @ B64, np.abs(A64) @ np.abs(B64))


def test_sum_over_batch_weight_gradient():
    # dW (Co x Ci) = sum_b D[b] (Co x P) X[b]^T (P x Ci), the operator's weight-gradient form
    rng = np.random.default_rng(11)
    batch, Co, Ci, P = 5, 32, 3, 20000
    D = rng.standard_normal((batch, Co, P)).astype(np.float32)
    X = rng.standard_normal((batch, Ci, P)).astype(np.float32)
    C = _run(D, X, np.full((Co, Ci), np.nan, np.float32), 1.0, 0.0, (P, 1, Co * P), (1, P, Ci * P), (Ci, 1, 0),
             batch, Co, Ci, P, split=True, sum_batch=True)
    D64, X64 = D.astype(np.float64), X.astype(np.float64)
    ref = np.einsum("bop,bip->oi", D64, X64)
    bound = np.einsum("bop,bip->oi", np.abs(D64), np.abs(X64))
    _check(C, ref, bound)


def test_empty_depth_scales_c():
    rng = np.random.default_rng(2)
    m, n = 50, 20
    C0 = rng.standard_normal((m, n)).astype(np.float32)
    A = np.zeros((m, 1), np.float32)
    B = np.zeros((1, n), np.float32)
    C = _run(A, B, C0, 1.0, 3.0, (1, 1, 0), (n, 1, 0), (n, 1, 0), 1, m, n, 0)
    np.testing.assert_array_equal(C, (3.0 * C0).astype(np.float32))


def test_deterministic():
    rng = np.random.default_rng(9)
    m, n, k = 64, 64, 30000
    A = rng.standard_normal((m, k)).astype(np.float32)
    B = rng.standard_normal((k, n)).astype(np.float32)
    runs = [_run(A, B, np.zeros((m, n), np.float32), 1.0, 0.0, (k, 1, 0), (n, 1, 0), (n, 1, 0), 1, m, n, k,
                 split=True) for _ in range(2)]
    np.testing.assert_array_equal(runs[0], runs[1])


def test_async_entry_matches_synchronous_one():
    # b200_tc_sgemm_async with a caller workspace and error word gives the synchronous entry's bits
    import torch

    rng = np.random.default_rng(21)
    batch, Co, Ci, P = 3, 32, 16, 30000
    D = rng.standard_normal((batch, Co, P)).astype(np.float32)
    X = rng.standard_normal((batch, Ci, P)).astype(np.float32)
    ref = _run(D, X, np.zeros((Co, Ci), np.float32), 1.0, 0.0, (P, 1, Co * P), (1, P, Ci * P), (Ci, 1, 0),
               batch, Co, Ci, P, split=True, sum_batch=True)
    Dd, Xd = _dev(D), _dev(X)
    C = torch.zeros((Co, Ci), dtype=torch.float32, device="cuda")
    ws = torch.empty(Co * Ci * batch * 64, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    S.tc_sgemm_async(batch, Co, Ci, P, 1.0, (Dd.data_ptr(), P, 1, Co * P), (Xd.data_ptr(), 1, P, Ci * P), 0.0,
                     (C.data_ptr(), Ci, 1, 0), ws.data_ptr(), ws.numel(), err.data_ptr(), sum_batch=True)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    np.testing.assert_array_equal(C.cpu().numpy(), ref)
