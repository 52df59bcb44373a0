"""Comparison helpers shared by the parity tests."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def bv_test1_fixture():
    """Fixture of src/sys/classes/bv/tests/test1.c:58-96 (n=10, k=5, l=3)."""
    n, k, l = 10, 5, 3
    X = np.zeros((n, k), order="F")
    for j in range(k):
        for i in range(4):
            if i + j < n:
                X[i + j, j] = 3 * i + j - 2
    Y = np.zeros((n, l), order="F")
    for j in range(l):
        Y[:, j] = (j + 1) / 4.0
    Q = np.array([[2.0 if i < j else -0.5 for j in range(l)] for i in range(k)], order="F")
    return X, Y, Q


def bv_test2_fixture(n=20, k=8):
    """Fixture of src/sys/classes/bv/tests/test2.c:55-62."""
    X = np.zeros((n, k), order="F")
    for j in range(k):
        for i in range(n // 2 + 1):
            if i + j < n:
                X[i + j, j] = (3.0 * i + j - 2) / (2 * (i + j + 1))
    return X


def ds_test2_matrix(n=12):
    A = np.zeros((n, n))
    for i in range(n):
        A[i, i] = 2.0
    for j in (1, 2):
        for i in range(n - j):
            A[i, i + j] = A[i + j, i] = 1.0
    return A


def eig_set_match(a, b, rtol):
    """Largest relative distance from each value of a to the nearest value of b."""
    a = np.asarray(a)
    b = np.asarray(b)
    if len(a) == 0:
        return 0.0
    d = np.abs(a[:, None] - b[None, :]) / np.maximum(np.abs(a[:, None]), 1e-300)
    return float(d.min(axis=1).max())


def clusters(values, rtol=1e-8):
    """Group sorted-by-position values into clusters of (relatively) equal values."""
    vals = np.asarray(values)
    used = np.zeros(len(vals), dtype=bool)
    out = []
    for i in range(len(vals)):
        if used[i]:
            continue
        idx = np.where(~used & (np.abs(vals - vals[i]) <= rtol * abs(vals[i])))[0]
        used[idx] = True
        out.append((float(vals[i]), idx))
    return out


def max_subspace_sine(Xa, Xb):
    """sin of the largest principal angle of span(Xa) inside span(Xb) (dim Xa <= dim Xb)."""
    Qa, _ = np.linalg.qr(Xa)
    Qb, _ = np.linalg.qr(Xb)
    R = Qa - Qb @ (Qb.T @ Qa)
    return float(np.linalg.norm(R, 2))


def eigenspace_sines(evals_a, Xa, evals_b, Xb, rtol=1e-8):
    """For each cluster of evals_a, the sine of the largest angle between the
    smaller and the larger of the two computed eigenspaces of that value."""
    out = []
    for lam, ia in clusters(evals_a, rtol):
        ib = np.where(np.abs(np.asarray(evals_b) - lam) <= rtol * abs(lam))[0]
        if len(ib) == 0:
            out.append((lam, np.inf))
            continue
        A, B = Xa[:, ia], Xb[:, ib]
        s = max_subspace_sine(A, B) if A.shape[1] <= B.shape[1] else max_subspace_sine(B, A)
        out.append((lam, s))
    return out
