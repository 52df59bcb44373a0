"""Learned warm start for the anisotropic-diffusion family: data pipeline, training and
evaluation around the neural-operator kernels (NeuralOperator, b200_neural_op_*).

The family is -div(kappa grad u) on an N x N cell grid with kappa = exp(Gaussian random field,
variance 1, correlation length uniform in [0.05, 0.2]) (problems.diffusion_problem).  Targets are
the nev lowest eigenvectors that the plain solver (GPU LOBPCG, Jacobi preconditioner, block nev,
tol 1e-8) computes for each training field; the trained network maps a new field to a block of
nev fields that becomes the solver's initial space (EPSSetInitialSpace), with the seeded random
block as the fallback.
"""
import time

import numpy as np

from . import problems as P

DEFAULT_DIMS = dict(width=32, modes=16, layers=4, hidden=64)


def features(kappa):
    """(3, N*N) float32: log kappa, and x, y of the cell centres (row-major cells)."""
    kap = np.asarray(kappa, dtype=np.float64)
    N = kap.shape[0]
    c = (np.arange(N) + 0.5) / N
    yy, xx = np.meshgrid(c, c, indexing="ij")
    return np.stack([np.log(kap), xx, yy]).reshape(3, N * N).astype(np.float32)


def init_params(N, width, modes, layers, hidden, nout, seed=0):
    """Seeded initial parameters in the layout of b200_neural_op_create: Gaussian pointwise weights
    scaled by 1/sqrt(fan-in), spectral weights uniform in [-1/W, 1/W], zero biases."""
    rng = np.random.default_rng(seed)
    W, M2 = width, modes * modes
    parts = [rng.standard_normal((W, 3)) / np.sqrt(3.0), np.zeros(W)]
    for _ in range(layers):
        parts += [rng.uniform(-1.0, 1.0, (W, W, M2)) / W, rng.standard_normal((W, W)) / np.sqrt(W), np.zeros(W)]
    parts += [rng.standard_normal((hidden, W)) / np.sqrt(W), np.zeros(hidden),
              rng.standard_normal((nout, hidden)) / np.sqrt(hidden), np.zeros(nout)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def solve_lowest(S, csr, nev=16, tol=1e-8, X0=None, max_it=100000, orthog_block=None, stats=False, timing=False):
    """The plain solver for the family: LOBPCG, smallest real, Jacobi preconditioner, block nev,
    optional initial block X0 (n x k), iteration cap max_it (LOBPCG's default cap, max(100,
    2n/ncv), stops long before these operators converge), optional BVOrthogBlockType of the
    blocks (S.BV.OrthogBlockType; Gram-Schmidt when None).  Returns values, vectors (n x nconv),
    iterations, seconds, and the solver's counters when stats is set (with per-phase times when
    timing is set; the phase edges then synchronise the stream)."""
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setType(S.EPS.Type.LOBPCG)
    E.setWhichEigenpairs(S.SMALLEST_REAL)
    E.setDimensions(nev, 0)
    E.setTolerances(tol, max_it)
    E.setPreconditioner(S.EPS.PCType.JACOBI)
    if orthog_block is not None:
        E.setBVOrthogonalizationBlock(orthog_block)
    if timing:
        E.setTiming(True)
    if X0 is not None:
        E.setInitialSpace(X0)
    t0 = time.perf_counter()
    E.solve()
    secs = time.perf_counter() - t0
    nconv = E.getConverged()
    pairs = [E.getEigenpair(i) for i in range(min(nconv, nev))]
    out = {"vals": np.array([p[0] for p in pairs]), "X": np.stack([p[1] for p in pairs], axis=1) if pairs else None,
           "its": E.getIterationNumber(), "reason": E.getConvergedReason(), "nconv": nconv, "seconds": secs,
           "max_error": max((E.computeError(i) for i in range(min(nconv, nev))), default=None)}
    if stats:
        out["stats"] = E.getStats()
    E.destroy()
    A.destroy()
    return out


def dataset(S, N, seeds, nev=16, orthog_block=None):
    """Features (len(seeds), 3, N*N) and targets (len(seeds), nev, N*N), float32, from plain solves
    (orthog_block: the BVOrthogBlockType of the solver's blocks, Gram-Schmidt when None)."""
    F, T, its = [], [], []
    for sd in seeds:
        csr, kappa, _ = P.diffusion_problem(N, int(sd))
        r = solve_lowest(S, csr, nev, orthog_block=orthog_block)
        if r["nconv"] < nev:
            raise RuntimeError(f"plain solve of field {sd} converged {r['nconv']} < {nev} pairs")
        X = r["X"] / np.linalg.norm(r["X"], axis=0)
        F.append(features(kappa))
        T.append(X.T.astype(np.float32))
        its.append(r["its"])
    return np.ascontiguousarray(np.stack(F)), np.ascontiguousarray(np.stack(T)), np.array(its)


def train(op, F, T, epochs, batch=8, lr=1e-3, seed=0, lr_final=None):
    """Adam over shuffled batches of the device tensors F, T; returns the mean loss of each epoch.
    With lr_final the step size decays geometrically from lr to lr_final over the epochs."""
    import torch

    rng = np.random.default_rng(seed)
    n = F.shape[0]
    hist = []
    for ep in range(epochs):
        step_lr = lr if lr_final is None else lr * (lr_final / lr) ** (ep / max(epochs - 1, 1))
        perm = rng.permutation(n)
        losses = []
        for i in range(0, n - batch + 1, batch):
            idx = torch.as_tensor(perm[i:i + batch], device=F.device)
            losses.append(op.trainStep(F.index_select(0, idx).contiguous(), T.index_select(0, idx).contiguous(),
                                       step_lr))
        hist.append(float(np.mean(losses)))
    return hist


def predict(op, F):
    """Network outputs for the device feature tensor F: numpy (batch, nout, N*N)."""
    return op.forward(F).cpu().numpy()


def captured(U, Y):
    """Fraction of the eigenvector subspace span(U) (n x k, orthonormal) captured by span(Y)."""
    Q, _ = np.linalg.qr(Y)
    return float(np.linalg.norm(U.T @ Q) ** 2 / U.shape[1])


def evaluate(S, op, N, seeds, nev=16):
    """Plain LOBPCG from the seeded random block against the learned block on each field: iterations,
    seconds, and the fraction of the converged eigenvectors the learned block already spans."""
    import torch

    rows = []
    for sd in seeds:
        csr, kappa, _ = P.diffusion_problem(N, int(sd))
        Fd = torch.from_numpy(features(kappa)[None]).cuda()
        Y = predict(op, Fd)[0].T.astype(np.float64)
        r0 = solve_lowest(S, csr, nev)
        r1 = solve_lowest(S, csr, nev, X0=Y)
        rows.append({"seed": int(sd), "its_random": r0["its"], "its_learned": r1["its"], "s_random": r0["seconds"],
                     "s_learned": r1["seconds"], "captured": captured(r0["X"], Y),
                     "converged": bool(r0["nconv"] >= nev and r1["nconv"] >= nev),
                     "max_error_learned": r1["max_error"]})
    return rows
