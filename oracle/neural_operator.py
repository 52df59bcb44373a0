"""CPU oracle (test infrastructure only) for the neural-operator kernels of
slepc_b200/csrc/learned.cu: the same network, loss and gradient restated in
numpy FP64, the backward pass derived by hand, layer by layer.  Only tests/
use it, as the checker of the GPU forward pass and gradients; its own
backward pass is pinned by central finite differences in
tests/test_learned_cpu.py.

Parameter layout (one flat array, the order of b200_neural_op_create):
  Pw (W x 3), Pb (W), then per layer l: R_l (W x W x M*M, index
  o*W*M*M + c*M*M + k*M + m), W_l (W x W), b_l (W); then Q1 (H x W), q1 (H),
  Q2 (K x H), q2 (K).  Activations are (batch, channels, N*N) with row-major
  cells.
"""
import math

import numpy as np
from scipy.special import erf


def sine_basis(N, M):
    i = np.arange(N)[:, None]
    k = np.arange(M)[None, :]
    return math.sqrt(2.0 / (N + 1)) * np.sin(np.pi * (i + 1) * (k + 1) / (N + 1))


def sizes(N, W, M, L, H, K):
    shapes = [("Pw", (W, 3)), ("Pb", (W,))]
    for l in range(L):
        shapes += [(f"R{l}", (W, W, M * M)), (f"W{l}", (W, W)), (f"b{l}", (W,))]
    shapes += [("Q1", (H, W)), ("q1", (H,)), ("Q2", (K, H)), ("q2", (K,))]
    return shapes


def unpack(theta, N, W, M, L, H, K):
    out, off = {}, 0
    for name, shp in sizes(N, W, M, L, H, K):
        n = int(np.prod(shp))
        out[name] = np.asarray(theta[off:off + n], dtype=np.float64).reshape(shp)
        off += n
    assert off == len(theta)
    return out


def pack(d, N, W, M, L, H, K):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in sizes(N, W, M, L, H, K)])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(theta, F, dims):
    """F: (B, 3, N*N).  Returns (Y, cache)."""
    N, W, M, L, H, K = dims
    p = unpack(theta, *dims)
    S = sine_basis(N, M)
    B = F.shape[0]
    v = np.einsum("oi,bip->bop", p["Pw"], F) + p["Pb"][None, :, None]
    cache = {"F": F, "V": [v], "U": [], "C": [], "S": S}
    for l in range(L):
        C = np.einsum("ik,bcij,jm->bckm", S, v.reshape(B, W, N, N), S).reshape(B, W, M * M)
        D = np.einsum("ocq,bcq->boq", p[f"R{l}"], C)
        s = np.einsum("ik,bokm,jm->boij", S, D.reshape(B, W, M, M), S).reshape(B, W, N * N)
        u = s + np.einsum("oc,bcp->bop", p[f"W{l}"], v) + p[f"b{l}"][None, :, None]
        cache["C"].append(C)
        cache["U"].append(u)
        v = gelu(u) if l < L - 1 else u
        cache["V"].append(v)
    z = np.einsum("hc,bcp->bhp", p["Q1"], v) + p["q1"][None, :, None]
    h = gelu(z)
    y = np.einsum("kh,bhp->bkp", p["Q2"], h) + p["q2"][None, :, None]
    cache.update(z=z, h=h)
    return y, cache


def loss(Y, T):
    """Mean over (b, k) of 1 - (y.u)^2 / (y.y); returns (loss, dL/dY)."""
    yu = np.einsum("bkp,bkp->bk", Y, T)
    yy = np.einsum("bkp,bkp->bk", Y, Y)
    n = Y.shape[0] * Y.shape[1]
    lval = float(np.mean(1.0 - yu * yu / yy))
    dY = (-2.0 * (yu / yy)[:, :, None] * T + 2.0 * (yu * yu / (yy * yy))[:, :, None] * Y) / n
    return lval, dY


def loss_grad(theta, F, T, dims):
    """Loss and gradient with respect to every parameter (flat, the layout above)."""
    N, W, M, L, H, K = dims
    p = unpack(theta, *dims)
    Y, c = forward(theta, F, dims)
    lval, dY = loss(Y, T)
    S = c["S"]
    B = F.shape[0]
    g = {}
    g["Q2"] = np.einsum("bkp,bhp->kh", dY, c["h"])
    g["q2"] = dY.sum(axis=(0, 2))
    dz = np.einsum("kh,bkp->bhp", p["Q2"], dY) * gelu_grad(c["z"])
    g["Q1"] = np.einsum("bhp,bcp->hc", dz, c["V"][L])
    g["q1"] = dz.sum(axis=(0, 2))
    dv = np.einsum("hc,bhp->bcp", p["Q1"], dz)
    for l in range(L - 1, -1, -1):
        du = dv * gelu_grad(c["U"][l]) if l < L - 1 else dv
        vin = c["V"][l]
        g[f"b{l}"] = du.sum(axis=(0, 2))
        g[f"W{l}"] = np.einsum("bop,bcp->oc", du, vin)
        dD = np.einsum("ik,boij,jm->bokm", S, du.reshape(B, W, N, N), S).reshape(B, W, M * M)
        g[f"R{l}"] = np.einsum("boq,bcq->ocq", dD, c["C"][l])
        dC = np.einsum("boq,ocq->bcq", dD, p[f"R{l}"])
        dv = (np.einsum("oc,bop->bcp", p[f"W{l}"], du)
              + np.einsum("ik,bckm,jm->bcij", S, dC.reshape(B, W, M, M), S).reshape(B, W, N * N))
    g["Pw"] = np.einsum("bop,bip->oi", dv, c["F"])
    g["Pb"] = dv.sum(axis=(0, 2))
    return lval, pack(g, *dims)
