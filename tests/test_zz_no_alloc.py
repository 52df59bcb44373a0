"""The allocation-free Gram-Schmidt entry point against the regular one.

b200_orthogonalize_column_noalloc serves callers that cannot allocate
device memory (their GPU memory belongs to a pool allocator, or they must
not grow the process's footprint); it takes its working memory from a fixed
array inside the library.  Two calls in a row, on different sizes, must each
give what b200_bv_orthogonalize_column gives on the same input -- the second
call proves that scratch left over from the first does not leak into it.
This file is collected last so that a failure here stops a -x run only after
every other test has run.
"""
import numpy as np
import pytest

import slepc_b200 as S

pytestmark = pytest.mark.gpu


def _case(n, j, m, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, j)))
    V = np.zeros((n, m), order="F")
    V[:, :j] = Q
    V[:, j] = Q @ (1e3 * rng.standard_normal(j)) + rng.standard_normal(n)  # forces the DGKS refinement
    return V


def _reference(V, j):
    n, m = V.shape
    bv = S.BV().create(n, m)
    bv.setColumns(V[:, : j + 1])
    H, nrm, lindep = bv.orthogonalizeColumn(j)
    col = bv.getColumn(j)
    bv.destroy()
    return H, nrm, lindep, col


def _noalloc(V, j):
    import torch

    n, m = V.shape
    ld = n + (n % 2)
    Vd = torch.zeros((m, ld), dtype=torch.float64, device="cuda")
    Vd[:, :n] = torch.from_numpy(np.ascontiguousarray(V.T))
    Hd = torch.full((j + 1,), np.nan, dtype=torch.float64, device="cuda")
    nrm, lindep = S.orthogonalize_column_noalloc(n, ld, m, Vd.data_ptr(), j, Hd.data_ptr())
    torch.cuda.synchronize()
    return Hd.cpu().numpy(), nrm, lindep, Vd[j, :n].cpu().numpy()


def test_noalloc_matches_regular_entry_point_twice():
    for n, j, m, seed in ((200003, 60, 62, 1), (4099, 17, 20, 2)):
        V = _case(n, j, m, seed)
        Hr, nr, lr, cr = _reference(V, j)
        Hn, nn, ln, cn = _noalloc(V, j)
        assert ln == lr
        np.testing.assert_allclose(nn, nr, rtol=1e-12)
        np.testing.assert_allclose(Hn, Hr, rtol=1e-11, atol=1e-13 * np.abs(Hr).max())
        np.testing.assert_allclose(cn, cr, rtol=0, atol=1e-12 * np.abs(cr).max())


def test_noalloc_matches_the_oracle():
    import oracle

    V = _case(30011, 24, 26, 3)
    Ho, no, lo = oracle.bv_orthogonalize_column(np.asfortranarray(V.copy()), 24)
    Hn, nn, ln, _ = _noalloc(V, 24)
    assert ln == lo
    np.testing.assert_allclose(nn, no, rtol=1e-12)
    np.testing.assert_allclose(Hn, Ho, rtol=1e-11, atol=1e-13 * np.abs(Ho).max())


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import torch

    # real (small) device buffers: only the argument check may run, and it must stop the call
    Vd = torch.zeros((300, 1000), dtype=torch.float64, device="cuda")
    Hd = torch.zeros(261, dtype=torch.float64, device="cuda")
    with pytest.raises(S.B200Error) as ei:
        S.orthogonalize_column_noalloc(1000, 1000, 300, Vd.data_ptr(), 260, Hd.data_ptr())
    assert ei.value.status == 1
    torch.cuda.synchronize()
