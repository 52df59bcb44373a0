"""Synthetic operators and start vectors for the Krylov-Schur workloads.

All matrices are returned as CSR triples (rowptr int32, colind int32,
values float64) with column indices sorted inside each row, which is what
PETSc's MatAssembly produces for MATSEQAIJ.
"""
import numpy as np


def laplacian_2d(n, m=None):
    """2-D 5-point Dirichlet Laplacian on an n x m grid in the ordering of
    SLEPc's ``src/eps/tutorials/ex2.c:46-53``: row II has i = II // n,
    j = II - i*n, diagonal 4 and -1 at II-n, II-1, II+1, II+n (when inside)."""
    m = n if m is None else m
    N = n * m
    II = np.arange(N, dtype=np.int64)
    i = II // n
    j = II - i * n
    cols, vals = [], []
    # sorted column order: II-n < II-1 < II < II+1 < II+n
    cols.append(np.where(i > 0, II - n, -1)); vals.append(-1.0)
    cols.append(np.where(j > 0, II - 1, -1)); vals.append(-1.0)
    cols.append(II); vals.append(4.0)
    cols.append(np.where(j < n - 1, II + 1, -1)); vals.append(-1.0)
    cols.append(np.where(i < m - 1, II + n, -1)); vals.append(-1.0)
    return _stack(N, cols, vals)


def laplacian_3d(nx, ny=None, nz=None):
    """3-D 7-point Dirichlet Laplacian on an nx x ny x nz grid, lexicographic
    ordering (x fastest): diagonal 6, -1 at +-1, +-nx, +-nx*ny."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    N = nx * ny * nz
    II = np.arange(N, dtype=np.int64)
    x = II % nx
    y = (II // nx) % ny
    z = II // (nx * ny)
    sxy = nx * ny
    cols, vals = [], []
    cols.append(np.where(z > 0, II - sxy, -1)); vals.append(-1.0)
    cols.append(np.where(y > 0, II - nx, -1)); vals.append(-1.0)
    cols.append(np.where(x > 0, II - 1, -1)); vals.append(-1.0)
    cols.append(II); vals.append(6.0)
    cols.append(np.where(x < nx - 1, II + 1, -1)); vals.append(-1.0)
    cols.append(np.where(y < ny - 1, II + nx, -1)); vals.append(-1.0)
    cols.append(np.where(z < nz - 1, II + sxy, -1)); vals.append(-1.0)
    return _stack(N, cols, vals)


def _stack(N, cols, vals):
    C = np.stack(cols, axis=1)
    Vv = np.broadcast_to(np.asarray(vals, dtype=np.float64), C.shape)
    mask = C >= 0
    counts = mask.sum(axis=1)
    rowptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    colind = C[mask].astype(np.int32)
    values = np.ascontiguousarray(Vv[mask], dtype=np.float64)
    return rowptr.astype(np.int32), colind, values


def laplacian_2d_eigs(n, m=None):
    m = n if m is None else m
    a = 2 - 2 * np.cos(np.pi * np.arange(1, n + 1) / (n + 1))
    b = 2 - 2 * np.cos(np.pi * np.arange(1, m + 1) / (m + 1))
    return (a[:, None] + b[None, :]).ravel()


def laplacian_3d_eigs(nx, ny=None, nz=None):
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    a = [2 - 2 * np.cos(np.pi * np.arange(1, k + 1) / (k + 1)) for k in (nx, ny, nz)]
    return (a[0][:, None, None] + a[1][None, :, None] + a[2][None, None, :]).ravel()


def laplacian_2d_eigenspace(lam, n, m=None, rtol=1e-10):
    """Orthonormal basis of the exact eigenspace of laplacian_2d(n, m) for eigenvalue lam
    (products of sines; entry II = i*n + j with j the fast index)."""
    m = n if m is None else m
    a = 2 - 2 * np.cos(np.pi * np.arange(1, n + 1) / (n + 1))
    b = 2 - 2 * np.cos(np.pi * np.arange(1, m + 1) / (m + 1))
    idx = np.argwhere(np.abs(a[:, None] + b[None, :] - lam) <= rtol * abs(lam))
    j = np.arange(n)
    i = np.arange(m)
    cols = []
    for p, q in idx:
        v = np.outer(np.sin(np.pi * (q + 1) * (i + 1) / (m + 1)), np.sin(np.pi * (p + 1) * (j + 1) / (n + 1))).ravel()
        cols.append(v / np.linalg.norm(v))
    return np.stack(cols, axis=1) if cols else np.zeros((n * m, 0))


def laplacian_3d_eigenspace(lam, nx, ny=None, nz=None, rtol=1e-10):
    """Orthonormal basis of the exact eigenspace of laplacian_3d for eigenvalue lam
    (products of sines; x is the fastest index)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    dims = (nx, ny, nz)
    ev = [2 - 2 * np.cos(np.pi * np.arange(1, k + 1) / (k + 1)) for k in dims]
    tot = ev[0][:, None, None] + ev[1][None, :, None] + ev[2][None, None, :]
    idx = np.argwhere(np.abs(tot - lam) <= rtol * abs(lam))
    cols = []
    for a, b, c in idx:
        sx = np.sin(np.pi * (a + 1) * np.arange(1, nx + 1) / (nx + 1))
        sy = np.sin(np.pi * (b + 1) * np.arange(1, ny + 1) / (ny + 1))
        sz = np.sin(np.pi * (c + 1) * np.arange(1, nz + 1) / (nz + 1))
        v = (sz[:, None, None] * sy[None, :, None] * sx[None, None, :]).ravel()
        cols.append(v / np.linalg.norm(v))
    return np.stack(cols, axis=1) if cols else np.zeros((nx * ny * nz, 0))


def start_vector(n, seed=0):
    """Seeded N(0,1) start vector (the EPSSetInitialSpace vector shared by the
    GPU path and the oracle)."""
    return np.random.default_rng(seed).standard_normal(n)


def to_scipy(csr, n=None):
    import scipy.sparse as sp

    rowptr, colind, vals = csr
    n = len(rowptr) - 1 if n is None else n
    return sp.csr_matrix((vals, colind, rowptr), shape=(n, n))


# ---------------------------------------------------------------- power-law rectangular matrix
_gen = None


def _genlib():
    global _gen
    if _gen is None:
        import ctypes

        from . import build as _b

        L = ctypes.CDLL(_b.build_generator())
        L.gen_powerlaw.restype = ctypes.c_int
        L.gen_powerlaw.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gen_uniform.restype = ctypes.c_double
        L.gen_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
        L.gen_normal.restype = ctypes.c_double
        L.gen_normal.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64]
        _gen = L
    return _gen


def powerlaw_rect(m, n, nnz_row=20, alpha=1.8, seed=0):
    """m x n CSR matrix with nnz_row distinct columns per row drawn from a power
    law with exponent alpha in the column index (few columns appear in almost
    every row) and N(0,1) values stored as float32: (rowptr, colind, vals)."""
    k = min(nnz_row, n)
    rowptr = np.empty(m + 1, dtype=np.int32)
    colind = np.empty(m * k, dtype=np.int32)
    vals = np.empty(m * k, dtype=np.float32)
    st = _genlib().gen_powerlaw(m, n, nnz_row, float(alpha), seed, rowptr.ctypes.data, colind.ctypes.data,
                                vals.ctypes.data)
    if st:
        raise ValueError("invalid power-law matrix parameters")
    return rowptr, colind, vals


def _mix(z):
    M = (1 << 64) - 1
    z = (z + 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def powerlaw_rect_py(m, n, nnz_row=20, alpha=1.8, seed=0):
    """Pure-Python restatement of powerlaw_rect for small sizes (checks the C generator)."""
    import math

    M = (1 << 64) - 1

    def bits(stream, row, t):
        return _mix(_mix((seed * 4 + stream) & M) ^ ((row << 24) ^ t))

    def uniform(stream, row, t):
        return (bits(stream, row, t) >> 11) * (1.0 / 9007199254740992.0)

    k = min(nnz_row, n)
    a1 = alpha - 1.0
    tail = 1.0 - math.pow(n + 1.0, -a1)
    rowptr = np.arange(m + 1, dtype=np.int32) * k
    colind = np.empty(m * k, dtype=np.int32)
    vals = np.empty(m * k, dtype=np.float32)
    for i in range(m):
        cols = []
        t = 0
        while len(cols) < k and t < (1 << 24):
            x = math.pow(1.0 - uniform(0, i, t) * tail, -1.0 / a1)
            c = min(max(int(math.floor(x)) - 1, 0), n - 1)
            if c not in cols:
                cols.append(c)
            t += 1
        c = 0
        while len(cols) < k and c < n:
            if c not in cols:
                cols.append(c)
            c += 1
        colind[i * k:(i + 1) * k] = sorted(cols)
        for j in range(k):
            u1 = ((bits(1, i, 2 * j) >> 11) + 1.0) * (1.0 / 9007199254740992.0)
            u2 = uniform(1, i, 2 * j + 1)
            vals[i * k + j] = np.float32(math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2))
    return rowptr, colind, vals


# ---------------------------------------------------------------- anisotropic diffusion (learned warm start workload)
def gaussian_random_field(N, corr_len, seed, variance=1.0):
    """N x N samples on the cell centres of the unit square of a stationary Gaussian field with
    squared-exponential covariance variance * exp(-r^2 / (2 corr_len^2)): white noise filtered
    spectrally on a 2N x 2N periodic grid (so the wrap-around correlation stays outside the
    square), then shifted and scaled to mean 0 and the given variance."""
    rng = np.random.default_rng(seed)
    M = 2 * N
    xi = rng.standard_normal((M, M))
    k = np.fft.fftfreq(M, d=1.0 / N)  # cycles per unit length
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    field = np.fft.ifft2(np.fft.fft2(xi) * np.exp(-np.pi ** 2 * corr_len ** 2 * k2)).real[:N, :N]
    field = field - field.mean()
    return field * np.sqrt(variance) / field.std()


def diffusion_fv(kappa):
    """5-point finite-volume matrix of -div(kappa grad u) on the N x N cell grid of the unit
    square with u = 0 on the boundary, multiplied by h^2: face coefficients are harmonic means
    of the two cell values, a boundary face contributes 2 kappa_cell.  Row-major cell
    ordering; returns (rowptr, colind, vals)."""
    kap = np.asarray(kappa, dtype=np.float64)
    N = kap.shape[0]
    idx = np.arange(N * N).reshape(N, N)
    hx = 2.0 * kap[:, :-1] * kap[:, 1:] / (kap[:, :-1] + kap[:, 1:])   # faces between (i,j) and (i,j+1)
    hy = 2.0 * kap[:-1, :] * kap[1:, :] / (kap[:-1, :] + kap[1:, :])   # faces between (i,j) and (i+1,j)
    diag = np.zeros((N, N))
    diag[:, :-1] += hx
    diag[:, 1:] += hx
    diag[:-1, :] += hy
    diag[1:, :] += hy
    diag[:, 0] += 2 * kap[:, 0]
    diag[:, -1] += 2 * kap[:, -1]
    diag[0, :] += 2 * kap[0, :]
    diag[-1, :] += 2 * kap[-1, :]
    rows = [idx.ravel(), idx[:, :-1].ravel(), idx[:, 1:].ravel(), idx[:-1, :].ravel(), idx[1:, :].ravel()]
    cols = [idx.ravel(), idx[:, 1:].ravel(), idx[:, :-1].ravel(), idx[1:, :].ravel(), idx[:-1, :].ravel()]
    vals = [diag.ravel(), -hx.ravel(), -hx.ravel(), -hy.ravel(), -hy.ravel()]
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rowptr = np.zeros(N * N + 1, dtype=np.int32)
    np.cumsum(np.bincount(r, minlength=N * N), out=rowptr[1:])
    return rowptr, c.astype(np.int32), v


def diffusion_problem(N, seed):
    """kappa = exp(GRF) with variance 1 and a correlation length drawn uniformly from
    [0.05, 0.2] (from the seed), and its finite-volume matrix: (csr, kappa, corr_len)."""
    rng = np.random.default_rng([seed, 0x4b])
    corr_len = float(rng.uniform(0.05, 0.2))
    kappa = np.exp(gaussian_random_field(N, corr_len, [seed, 0x47]))
    return diffusion_fv(kappa), kappa, corr_len


# ---------------------------------------------------------------- k-NN graph batches (batched workload)
def _knnlib():
    import ctypes

    L = _genlib()
    if not hasattr(L, "_knn_ready"):
        L.knn_build.restype = ctypes.c_int64
        L.knn_build.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.knn_points.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_void_p]
        L.knn_build_batch.restype = ctypes.c_int
        L.knn_build_batch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
        L._knn_ready = True
    return L


def knn_operator(n, k=8, seed=0, problem=0):
    """2I - L_norm of the symmetrised k-NN graph of n random points (problem `problem` of the
    batch with this seed): (rowptr, colind, vals)."""
    L = _knnlib()
    cap = n * (4 * k + 2)
    while True:
        rowptr = np.empty(n + 1, dtype=np.int32)
        colind = np.empty(cap, dtype=np.int32)
        vals = np.empty(cap)
        nnz = L.knn_build(n, k, seed, problem, rowptr.ctypes.data, colind.ctypes.data, vals.ctypes.data, cap)
        if nnz < 0:
            raise ValueError("invalid k-NN parameters")
        if nnz <= cap:
            return rowptr, colind[:nnz].copy(), vals[:nnz].copy()
        cap = int(nnz)


def knn_points(n, seed=0, problem=0):
    xy = np.empty(2 * n)
    _knnlib().knn_points(n, seed, problem, xy.ctypes.data)
    return xy.reshape(n, 2)


def batch_sizes(nprob, seed=0, lo=500, hi=20000):
    """Problem sizes n ~ U[lo, hi] (integers, inclusive) from the seed."""
    return np.random.default_rng([seed, 0x5a]).integers(lo, hi + 1, size=nprob).astype(np.int32)


class Batch:
    """Concatenated CSR of a batch: problem p has rows [row_off[p], row_off[p] + ns[p]) of the
    batch, its own row pointer at rowptr[row_off[p] + p : row_off[p] + p + ns[p] + 1] (local
    offsets from nnz_off[p]) and local column indices."""

    def __init__(self, ns, rowptr, colind, vals, row_off, nnz_off):
        self.ns, self.rowptr, self.colind, self.vals = ns, rowptr, colind, vals
        self.row_off, self.nnz_off = row_off, nnz_off

    @property
    def nprob(self):
        return len(self.ns)

    def problem(self, p):
        r0 = int(self.row_off[p]) + p
        n = int(self.ns[p])
        z0, z1 = int(self.nnz_off[p]), int(self.nnz_off[p + 1])
        return self.rowptr[r0:r0 + n + 1].copy(), self.colind[z0:z1].copy(), self.vals[z0:z1].copy()

    def subset(self, idx):
        """The batch of problems idx (in that order), with the same per-problem arrays."""
        idx = [int(p) for p in idx]
        ns = self.ns[idx].astype(np.int32) if idx else np.zeros(0, dtype=np.int32)
        parts = [self.problem(p) for p in idx]
        row_off = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum(ns, out=row_off[1:])
        nnz_off = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum([len(c) for _, c, _ in parts], out=nnz_off[1:])
        cat = (lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dtype=dt))
        return Batch(ns, cat([r for r, _, _ in parts], np.int32), cat([c for _, c, _ in parts], np.int32),
                     cat([v for _, _, v in parts], np.float64), row_off, nnz_off)

    def rows_of(self, x, idx):
        """The slices of a batch-long vector x (sum of ns entries) that belong to problems idx."""
        xs = [x[int(self.row_off[p]):int(self.row_off[p + 1])] for p in idx]
        return np.concatenate(xs) if xs else np.zeros(0, dtype=x.dtype)


def knn_batch(ns, k=8, seed=0):
    """The batch of k-NN operators for sizes ns (OpenMP over problems)."""
    L = _knnlib()
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    nprob = len(ns)
    counts = np.zeros(nprob, dtype=np.int64)
    if L.knn_build_batch(nprob, ns.ctypes.data, k, seed, counts.ctypes.data, None, None, None, None, None):
        raise ValueError("invalid k-NN parameters")
    row_off = np.zeros(nprob + 1, dtype=np.int64)
    np.cumsum(ns, out=row_off[1:])
    nnz_off = np.zeros(nprob + 1, dtype=np.int64)
    np.cumsum(counts, out=nnz_off[1:])
    rowptr = np.zeros(int(row_off[-1]) + nprob, dtype=np.int32)
    colind = np.zeros(int(nnz_off[-1]), dtype=np.int32)
    vals = np.zeros(int(nnz_off[-1]))
    if L.knn_build_batch(nprob, ns.ctypes.data, k, seed, counts.ctypes.data, row_off.ctypes.data, nnz_off.ctypes.data,
                         rowptr.ctypes.data, colind.ctypes.data, vals.ctypes.data):
        raise RuntimeError("k-NN batch build failed")
    return Batch(ns, rowptr, colind, vals, row_off, nnz_off)
