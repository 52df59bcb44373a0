"""The neural-operator warm start on the GPU.

* Forward pass, loss and the gradient of every parameter tensor from the library's own FP32
  kernels against the FP64 numpy oracle (itself pinned by finite differences): outputs and loss
  to 1e-4 relative, each gradient tensor to 2e-3 relative in norm (FP32 sums over the grid).
* Training with those kernels lowers the loss on eigenvectors computed by the plain solver.
* On fields the network never saw, LOBPCG started from the network's block takes fewer
  iterations than from the seeded random block, and still converges every pair to 1e-8.
"""
import numpy as np
import pytest

import slepc_b200 as S
from oracle import neural_operator as NO
from slepc_b200 import learned as L
from slepc_b200 import problems as P

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


@pytest.mark.parametrize("dims,B", [((16, 8, 6, 2, 16, 4), 3), ((12, 4, 5, 3, 8, 5), 2)])
def test_forward_loss_and_gradients_vs_oracle(dims, B):
    torch = _torch()
    rng = np.random.default_rng(sum(dims))
    N, W, M, Ly, H, K = dims
    theta = L.init_params(*dims, seed=4)
    theta = (theta + 0.05 * rng.standard_normal(theta.size)).astype(np.float32)
    F = rng.standard_normal((B, 3, N * N)).astype(np.float32)
    T = rng.standard_normal((B, K, N * N))
    T = (T / np.linalg.norm(T, axis=2, keepdims=True)).astype(np.float32)
    op = S.NeuralOperator().create(*dims)
    op.setParams(theta)
    Fd, Td = torch.from_numpy(F).cuda(), torch.from_numpy(T).cuda()
    Y = op.forward(Fd).cpu().numpy()
    Yo, _ = NO.forward(theta.astype(np.float64), F.astype(np.float64), dims)
    assert np.linalg.norm(Y - Yo) <= 1e-4 * np.linalg.norm(Yo)
    lo, go = NO.loss_grad(theta.astype(np.float64), F.astype(np.float64), T.astype(np.float64), dims)
    lg, gg = op.lossGrad(Fd, Td)
    assert abs(lg - lo) <= 1e-4 * abs(lo)
    off = 0
    for name, shp in NO.sizes(*dims):
        n = int(np.prod(shp))
        a, b = gg[off:off + n], go[off:off + n]
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-9, (name, np.linalg.norm(a - b), np.linalg.norm(b))
        off += n
    assert np.allclose(op.getParams(), theta)
    op.destroy()


def test_training_lowers_the_loss_on_solver_eigenvectors():
    torch = _torch()
    N, nev = 16, 4
    F, T, _ = L.dataset(S, N, range(24), nev)
    Fd, Td = torch.from_numpy(F).cuda(), torch.from_numpy(T).cuda()
    dims = (N, 8, 6, 3, 16, nev)
    op = S.NeuralOperator().create(*dims)
    op.setParams(L.init_params(*dims, seed=0))
    before = op.loss(Fd, Td)
    hist = L.train(op, Fd, Td, epochs=60, batch=8, lr=2e-3)
    after = op.loss(Fd, Td)
    assert after < 0.5 * before, (before, after, hist[-5:])
    op.destroy()


def test_strided_tensors_are_read_as_their_values():
    """A non-contiguous targets tensor gives the loss of its values (the wrapper densifies it)."""
    torch = _torch()
    rng = np.random.default_rng(5)
    dims = (8, 4, 3, 2, 6, 3)
    op = S.NeuralOperator().create(*dims)
    op.setParams(L.init_params(*dims, seed=1))
    F = torch.from_numpy(rng.standard_normal((2, 3, 64)).astype(np.float32)).cuda()
    T = rng.standard_normal((2, 64, 3)).astype(np.float32).transpose(0, 2, 1)  # strided view
    Td = torch.from_numpy(T).cuda()
    assert not Td.is_contiguous()
    assert op.loss(F, Td) == op.loss(F, Td.contiguous())
    op.destroy()


def test_learned_start_saves_lobpcg_iterations_on_new_fields():
    """Train on the plain solver's eigenvectors of 64 fields (32 x 32 grid, 8 lowest), then solve 8
    fields the network never saw from the seeded random block and from the network's block."""
    torch = _torch()
    N, nev = 32, 8
    F, T, _ = L.dataset(S, N, range(64), nev)
    Fd, Td = torch.from_numpy(F).cuda(), torch.from_numpy(T).cuda()
    dims = (N, 16, 8, 4, 32, nev)
    op = S.NeuralOperator().create(*dims)
    op.setParams(L.init_params(*dims, seed=0))
    hist = L.train(op, Fd, Td, epochs=150, batch=8, lr=2e-3, lr_final=2e-4)
    assert hist[-1] < 0.5 * hist[0]
    rows = L.evaluate(S, op, N, range(20000, 20008), nev)
    assert all(r["converged"] and r["max_error_learned"] <= 1e-8 for r in rows)
    its_r = np.mean([r["its_random"] for r in rows])
    its_l = np.mean([r["its_learned"] for r in rows])
    assert its_l < its_r, (its_l, its_r, rows)
    assert np.mean([r["captured"] for r in rows]) > 0.3
    op.destroy()
