"""CPU oracle for the Hermitian Krylov-Schur path -- test infrastructure only.

This package is the checker: it restates SLEPc's Krylov-Schur / BV / DS
arithmetic in plain C (``ks_oracle.c``) and exposes it to Python through
ctypes.  Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` may import it.  The product library never links or calls it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

LARGEST_MAGNITUDE, SMALLEST_MAGNITUDE, LARGEST_REAL, SMALLEST_REAL = 1, 2, 3, 4
ORTHOG_BLOCK_GS, ORTHOG_BLOCK_CHOL, ORTHOG_BLOCK_SVQB = 0, 1, 4  # BVOrthogBlockType
CONVERGED_TOL, DIVERGED_ITS, DIVERGED_BREAKDOWN, ITERATING = 1, -1, -2, 0

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        L.oracle_eps_solve.restype = ctypes.c_int
        L.oracle_eps_solve.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _dp, _dp, _dp, _ip]
        L.oracle_bv_orthogonalize_column.argtypes = [ctypes.c_int] * 3 + [_dp, ctypes.c_int, _dp, _dp, _ip]
        L.oracle_bv_orthonormalize_column.argtypes = [ctypes.c_int] * 3 + [_dp, ctypes.c_int, _dp, _dp, _ip]
        L.oracle_bv_orthogonalize_vec.argtypes = [ctypes.c_int] * 3 + [_dp, _dp, _dp, _dp, _ip]
        L.oracle_bv_multinplace.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _dp,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_ds_hep_dense.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp]
        L.oracle_ds_hep_compact.argtypes = [ctypes.c_int] * 6 + [_dp, _dp, _dp, _dp]
        L.oracle_residual.restype = ctypes.c_double
        L.oracle_residual.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, ctypes.c_double]
        L.oracle_spmv.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, _dp]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_lobpcg.restype = ctypes.c_int
        L.oracle_lobpcg.argtypes = [ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, _ip]
        L.oracle_bv_orthogonalize_block.restype = ctypes.c_int
        L.oracle_bv_orthogonalize_block.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, _dp, ctypes.c_int]
        L.oracle_eps_solve_batch.restype = ctypes.c_int
        L.oracle_eps_solve_batch.argtypes = [ctypes.c_int, _ip, _ip, _ip, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, _dp, _ip]
        L.oracle_csr_transpose.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _ip, _ip, _dp]
        L.oracle_svd_cross.restype = ctypes.c_int
        L.oracle_svd_cross.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _ip, _ip, _dp, _dp,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _ip]
        L.oracle_random_entry.restype = ctypes.c_double
        L.oracle_random_entry.argtypes = [ctypes.c_uint64] * 3
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def set_threads(n):
    lib().oracle_set_threads(int(n))


def set_locking(lock):
    """EPSKrylovSchurSetLocking for the oracle's Krylov-Schur (process-wide; True by default)."""
    lib().oracle_set_locking(1 if lock else 0)


def spmv(A, x):
    rowptr, colind, vals = _csr(A)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(A.shape[0])
    lib().oracle_spmv(A.shape[0], _i(rowptr), _i(colind), _d(vals), _d(x), _d(y))
    return y


def _csr(A):
    return (np.ascontiguousarray(A.indptr, dtype=np.int32), np.ascontiguousarray(A.indices, dtype=np.int32),
            np.ascontiguousarray(A.data, dtype=np.float64))


class SolveResult:
    def __init__(self, evals, X, errest, nconv, its, reason, lanczos_steps, restarts, column_visits):
        self.evals, self.X, self.errest = evals, X, errest
        self.nconv, self.its, self.reason = nconv, its, reason
        self.lanczos_steps, self.restarts, self.column_visits = lanczos_steps, restarts, column_visits


def eps_solve(A, v0, nev, ncv, tol=1e-8, which=LARGEST_MAGNITUDE, mpd=0, max_it=0, max_restarts=0, want_vectors=True):
    """EPSSolve with EPSKRYLOVSCHUR on a symmetric scipy CSR matrix A."""
    n = A.shape[0]
    rowptr, colind, vals = _csr(A)
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    evals = np.zeros(ncv + 1)
    errest = np.zeros(ncv + 1)
    X = np.zeros((ncv + 1, n)) if want_vectors else None
    info = np.zeros(8, dtype=np.int32)
    st = lib().oracle_eps_solve(n, _i(rowptr), _i(colind), _d(vals), _d(v0), nev, ncv, mpd, tol, max_it, which,
                                max_restarts, _d(evals), _d(X) if want_vectors else None, _d(errest), _i(info))
    if st:
        raise RuntimeError(f"oracle_eps_solve failed with status {st}")
    nconv = int(info[0])
    return SolveResult(evals[:nconv].copy(), X[:nconv].T.copy() if want_vectors else None, errest[:nconv].copy(),
                       nconv, int(info[1]),
                       int(info[2]), int(info[3]), int(info[4]), int(info[5]))


def bv_orthogonalize_column(V, j, normalize=False):
    """BVOrthogonalizeColumn / BVOrthonormalizeColumn on a Fortran-ordered n x m array (in place)."""
    assert V.flags.f_contiguous and V.dtype == np.float64
    n, m = V.shape
    H = np.zeros(j + 1)
    nrm = ctypes.c_double()
    lnd = ctypes.c_int()
    f = lib().oracle_bv_orthonormalize_column if normalize else lib().oracle_bv_orthogonalize_column
    st = f(n, m, n, _d(V), j, _d(H), ctypes.byref(nrm), ctypes.byref(lnd))
    if st:
        raise RuntimeError(f"orthogonalize column failed {st}")
    return H, nrm.value, bool(lnd.value)


def bv_orthogonalize_vec(V, k, v):
    assert V.flags.f_contiguous
    n = V.shape[0]
    v = np.array(v, dtype=np.float64)
    H = np.zeros(max(k, 1))
    nrm = ctypes.c_double()
    lnd = ctypes.c_int()
    st = lib().oracle_bv_orthogonalize_vec(n, k, n, _d(V), _d(v), _d(H), ctypes.byref(nrm), ctypes.byref(lnd))
    if st:
        raise RuntimeError(f"orthogonalize vec failed {st}")
    return v, H[:k], nrm.value, bool(lnd.value)


def bv_orthogonalize_block(V, l, k, block_type):
    """BVOrthogonalize of columns [l,k) of a Fortran-ordered n x m array (in place) with block
    type ORTHOG_BLOCK_CHOL or ORTHOG_BLOCK_SVQB; returns R (k x k) with V_in = V_out R on [0,k)."""
    assert V.flags.f_contiguous and V.dtype == np.float64
    n = V.shape[0]
    R = np.zeros((k, k), order="F")
    st = lib().oracle_bv_orthogonalize_block(n, n, _d(V), l, k, block_type, _d(R), k)
    if st:
        raise RuntimeError(f"orthogonalize block failed {st}")
    return R


def bv_multinplace(V, l, k, Q, s, e):
    assert V.flags.f_contiguous and Q.flags.f_contiguous
    n = V.shape[0]
    lib().oracle_bv_multinplace(n, n, _d(V), l, k, _d(Q), Q.shape[0], s, e)


def ds_hep_dense(A, which=LARGEST_MAGNITUDE, ld=None):
    n = A.shape[0]
    ld = ld or n
    Af = np.zeros((ld, ld), order="F")
    Af[:n, :n] = A
    Q = np.zeros((ld, ld), order="F")
    wr = np.zeros(ld)
    st = lib().oracle_ds_hep_dense(n, ld, _d(Af), which, _d(wr), _d(Q))
    if st:
        raise RuntimeError(f"ds_hep_dense failed {st}")
    return wr[:n], Q[:n, :n]


def residual(A, x, lam):
    rowptr, colind, vals = _csr(A)
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oracle_residual(A.shape[0], _i(rowptr), _i(colind), _d(vals), _d(x), float(lam))


def random_entry(seed, stream, i):
    return lib().oracle_random_entry(seed, stream, i)


def csr_transpose(rowptr, colind, vals, shape):
    """Explicit transpose (MatTranspose_SeqAIJ order) of CSR arrays; returns (rowptr_t, colind_t, vals_t)."""
    m, n = shape
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    colind = np.ascontiguousarray(colind, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nnz = int(rowptr[m])
    rt = np.zeros(n + 1, dtype=np.int32)
    ct = np.zeros(max(nnz, 1), dtype=np.int32)
    vt = np.zeros(max(nnz, 1))
    lib().oracle_csr_transpose(m, n, _i(rowptr), _i(colind), _d(vals), _i(rt), _i(ct), _d(vt))
    return rt, ct[:nnz], vt[:nnz]


class SVDResult:
    def __init__(self, sigma, U, V, rel_error, nconv, its, reason, lanczos_steps, restarts, column_visits):
        self.sigma, self.U, self.V, self.rel_error = sigma, U, V, rel_error
        self.nconv, self.its, self.reason = nconv, its, reason
        self.lanczos_steps, self.restarts, self.column_visits = lanczos_steps, restarts, column_visits


def svd_cross(rowptr, colind, vals, shape, v0, nsv, ncv, tol=0.0, largest=True, mpd=0, max_it=0, max_restarts=0):
    """SVDSolve with SVDCROSS on an m x n CSR matrix (values as float64; FP32-stored
    matrices pass their float32 values widened).  For m < n the transpose is
    solved and U, V swapped back, as SVDSetUp / SVDGetSingularTriplet do; v0 then
    has length m."""
    m, n = shape
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    colind = np.ascontiguousarray(colind, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    rt, ct, vt = csr_transpose(rowptr, colind, vals, shape)
    swapped = m < n
    if swapped:
        rowptr, colind, vals, rt, ct, vt = rt, ct, vt, rowptr, colind, vals
        m, n = n, m
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    assert v0.shape == (n,)
    sig = np.zeros(ncv + 1)
    U = np.zeros((ncv + 1, m))
    V = np.zeros((ncv + 1, n))
    err = np.zeros(ncv + 1)
    info = np.zeros(8, dtype=np.int32)
    st = lib().oracle_svd_cross(m, n, _i(rowptr), _i(colind), _d(vals), _i(rt), _i(ct), _d(vt), _d(v0), nsv, ncv,
                                mpd, tol, max_it, 0 if largest else 1, max_restarts, _d(sig), _d(U), _d(V),
                                _d(err), _i(info))
    if st:
        raise RuntimeError(f"oracle_svd_cross failed with status {st}")
    k = int(info[0])
    U, V = U[:k].T.copy(), V[:k].T.copy()
    if swapped:
        U, V = V, U
    return SVDResult(sig[:k].copy(), U, V, err[:k].copy(), k, int(info[1]), int(info[2]), int(info[3]),
                     int(info[4]), int(info[5]))


def lobpcg(A, nev, bs=0, ncv=0, tol=1e-8, max_it=0, which=SMALLEST_REAL, pc="jacobi", lock=True, restart=0.9,
           X0=None, orthog_block=ORTHOG_BLOCK_GS):
    """EPSSolve with EPSLOBPCG on a symmetric scipy CSR matrix; X0 (n x k) an initial space;
    orthog_block the BVOrthogBlockType of the blocks (ORTHOG_BLOCK_GS, _CHOL or _SVQB)."""
    n = A.shape[0]
    rowptr, colind, vals = _csr(A)
    cap = max(ncv, 3 * max(bs, min(16, nev)), ((nev - 1) // max(bs or min(16, nev), 1) + 3) * max(bs or min(16, nev), 1)) + 48
    evals = np.zeros(cap)
    errest = np.zeros(cap)
    X = np.zeros((cap, n))
    info = np.zeros(8, dtype=np.int32)
    nini = 0
    x0p = None
    if X0 is not None:
        X0 = np.asfortranarray(X0, dtype=np.float64)
        nini = X0.shape[1]
        x0p = _d(X0)
    st = lib().oracle_lobpcg(n, _i(rowptr), _i(colind), _d(vals), nev, bs, ncv, tol, max_it, which,
                             {"none": 0, "jacobi": 1}[pc], 1 if lock else 0, restart, orthog_block, x0p, nini,
                             _d(evals), _d(X),
                             _d(errest), _i(info))
    if st:
        raise RuntimeError(f"oracle_lobpcg failed with status {st}")
    k = int(info[0])
    return SolveResult(evals[:k].copy(), X[:k].T.copy(), errest[:k].copy(), k, int(info[1]), int(info[2]), 0, 0, 0)


def eps_solve_batch(ns, rowptr, colind, vals, v0, nev, ncv, tol=1e-8, which=LARGEST_REAL, threads=0):
    """oracle_eps_solve on every problem of a batch in parallel over problems: (evals (nprob x ncv), info (nprob x 6))."""
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    nprob = len(ns)
    evals = np.zeros((nprob, ncv))
    info = np.zeros((nprob, 6), dtype=np.int32)
    if threads:
        set_threads(threads)
    bad = lib().oracle_eps_solve_batch(nprob, _i(ns), _i(np.ascontiguousarray(rowptr, dtype=np.int32)),
                                       _i(np.ascontiguousarray(colind, dtype=np.int32)),
                                       _d(np.ascontiguousarray(vals, dtype=np.float64)),
                                       _d(np.ascontiguousarray(v0, dtype=np.float64)), nev, ncv, tol, which,
                                       _d(evals), _i(info))
    if bad:
        raise RuntimeError(f"{bad} oracle batch problems failed")
    return evals, info
