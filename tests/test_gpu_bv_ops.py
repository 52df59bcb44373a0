"""BV operations a SLEPc adapter fills into the BVOps table, through the C ABI.

* b200_bv_gram_schmidt is the gramschmidt op (include/slepc/private/bvimpl.h:53).
  BVOrthogonalizeGS's DGKS loop (src/sys/classes/bv/interface/bvorthog.c:174-203)
  is restated here on the host, calling it 1-3 times exactly as the reference
  calls BVOrthogonalizeGS1; the coefficients, norm and lindep flag must equal
  b200_bv_orthogonalize_column's (the fused device loop) and the oracle's.
* resize, copy, normalize and the transposed in-place product against numpy.
"""
import numpy as np
import pytest

import oracle
import slepc_b200 as S

pytestmark = pytest.mark.gpu

ETA = 0.7071  # bvfunc.c:178


def _basis(n, j, m, seed, mode):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, j)))
    V = np.zeros((n, m), order="F")
    V[:, :j] = Q
    if mode == "refine":  # mostly inside span(Q): the first pass leaves |v'| < eta |v|
        V[:, j] = Q @ (1e3 * rng.standard_normal(j)) + rng.standard_normal(n)
    elif mode == "dependent":  # in span(Q) up to rounding: lindep after three passes
        V[:, j] = Q @ rng.standard_normal(j)
    else:
        V[:, j] = rng.standard_normal(n)
    return V


def _bv(V, j):
    n, m = V.shape
    bv = S.BV().create(n, m)
    bv.setColumns(V[:, : j + 1])
    return bv


def _dgks_host(bv, j):
    """BVOrthogonalizeGS with BV_ORTHOG_REFINE_IFNEEDED and CGS, on the gramschmidt op."""
    import torch

    h = torch.zeros(j + 1, dtype=torch.float64, device="cuda")
    c = torch.zeros(j + 1, dtype=torch.float64, device="cuda")
    onrm, nrm = bv.gramSchmidt(j, None, h.data_ptr(), c.data_ptr())
    passes = 1
    while passes < 3 and nrm != 0.0 and abs(nrm) < ETA * abs(onrm):
        passes += 1
        onrm, nrm = bv.gramSchmidt(j, None, h.data_ptr(), c.data_ptr())
    lindep = not (nrm != 0.0 and abs(nrm) >= ETA * abs(onrm))
    H = h.cpu().numpy()
    H[j] = 0.0 if lindep else nrm  # BV_SetValue(bv,k,k,h,...)
    return H, nrm, lindep, passes


@pytest.mark.parametrize("mode", ["plain", "refine", "dependent"])
@pytest.mark.parametrize("n,j", [(50021, 37), (2001, 5)])
def test_gram_schmidt_op_in_the_reference_dgks_loop(mode, n, j):
    V = _basis(n, j, j + 3, n + j, mode)
    bv = _bv(V, j)
    Hh, nh, lh, passes = _dgks_host(bv, j)
    col_h = bv.getColumn(j)
    bv.destroy()
    bv = _bv(V, j)
    Hf, nf, lf = bv.orthogonalizeColumn(j)
    col_f = bv.getColumn(j)
    bv.destroy()
    Ho, no, lo = oracle.bv_orthogonalize_column(np.asfortranarray(V.copy()), j)
    assert lh == lf == lo
    if mode == "refine":
        assert passes >= 2
    scale = np.abs(Ho).max()
    np.testing.assert_allclose(Hh, Hf, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(Hh, Ho, rtol=0, atol=1e-11 * scale)
    if mode != "dependent":
        np.testing.assert_allclose(nh, no, rtol=1e-11)
        np.testing.assert_allclose(col_h, col_f, rtol=0, atol=1e-11 * np.abs(col_f).max())


def test_gram_schmidt_op_vector_variant_and_coefficients():
    import torch

    n, k = 30011, 12
    rng = np.random.default_rng(4)
    Q, _ = np.linalg.qr(rng.standard_normal((n, k)))
    bv = S.BV().create(n, k + 1)
    bv.setColumns(Q)
    bv.setActiveColumns(0, k)
    x = rng.standard_normal(n) + Q @ rng.standard_normal(k)
    v = torch.from_numpy(x.copy()).cuda()
    c = torch.zeros(k + 1, dtype=torch.float64, device="cuda")
    h = torch.full((k + 1,), 0.5, dtype=torch.float64, device="cuda")
    onrm, nrm = bv.gramSchmidt(0, v.data_ptr(), h.data_ptr(), c.data_ptr())
    cref = Q.T @ x
    np.testing.assert_allclose(c.cpu().numpy()[:k], cref, rtol=1e-12, atol=1e-12 * np.abs(cref).max())
    np.testing.assert_allclose(c.cpu().numpy()[k], x @ x, rtol=1e-12)
    np.testing.assert_allclose(h.cpu().numpy()[:k], 0.5 + cref, rtol=1e-12, atol=1e-12)
    assert h.cpu().numpy()[k] == 0.5  # only the k coefficients are accumulated
    np.testing.assert_allclose(onrm, np.linalg.norm(x), rtol=1e-12)
    w = x - Q @ cref
    np.testing.assert_allclose(v.cpu().numpy(), w, rtol=0, atol=1e-11 * np.abs(x).max())
    np.testing.assert_allclose(nrm, np.linalg.norm(w), rtol=1e-8)
    # no norms requested: no synchronisation, same update
    v2 = torch.from_numpy(x.copy()).cuda()
    assert bv.gramSchmidt(0, v2.data_ptr(), None, None, norms=False) is None
    np.testing.assert_allclose(v2.cpu().numpy(), w, rtol=0, atol=1e-11 * np.abs(x).max())
    bv.destroy()


def test_resize_copy_normalize_and_transposed_product():
    n, m = 4099, 6
    rng = np.random.default_rng(9)
    X = rng.standard_normal((n, m))
    bv = S.BV().create(n, m)
    bv.setColumns(X)
    bv.resize(9, copy=True)
    assert bv.getSizes()[1] == 9
    np.testing.assert_array_equal(bv.getColumns(m), X)
    bv.resize(4, copy=True)
    np.testing.assert_array_equal(bv.getColumns(4), X[:, :4])
    assert bv.getActiveColumns() == (0, 4)
    # BVCopy: active columns [1, 4) into Y from its column 2
    bv.setActiveColumns(1, 4)
    Y = S.BV().create(n, 6)
    Y.setActiveColumns(2, 6)
    bv.copy(Y)
    np.testing.assert_array_equal(Y.getColumns(5)[:, 2:5], X[:, 1:4])
    # BVNormalize
    Y.setActiveColumns(2, 5)
    nrm = Y.normalize()
    np.testing.assert_allclose(nrm, np.linalg.norm(X[:, 1:4], axis=0), rtol=1e-13)
    np.testing.assert_allclose(np.linalg.norm(Y.getColumns(5)[:, 2:5], axis=0), 1.0, rtol=1e-14)
    Y.destroy()
    # BVMultInPlaceHermitianTranspose: V(:, 1:3) = V(:, 0:4) Q(1:3, 0:4)^T
    bv.setActiveColumns(0, 4)
    Qm = rng.standard_normal((5, 4))
    V0 = bv.getColumns(4)
    bv.multInPlaceTranspose(Qm, 1, 3)
    got = bv.getColumns(4)
    np.testing.assert_allclose(got[:, 1:3], V0 @ Qm[1:3, :].T, rtol=1e-13, atol=1e-13)
    np.testing.assert_array_equal(got[:, [0, 3]], V0[:, [0, 3]])
    bv.destroy()
