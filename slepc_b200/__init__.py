"""B200-native Hermitian Krylov-Schur eigensolver (SLEPc's EPSKRYLOVSCHUR inner loop).

Python mirror of the C ABI in ``include/slepc_b200.h``.  Class and method
names follow slepc4py (``EPS.setOperators``, ``setProblemType``,
``setDimensions``, ``setTolerances``, ``setWhichEigenpairs``,
``setInitialSpace``, ``solve``, ``getConverged``, ``getEigenpair``,
``computeError`` ...; ``BV.orthogonalizeColumn``, ``multInPlace`` ...), so code
written against SLEPc reads the same.  Every call goes to the CUDA library
``libslepc_b200.so``; there is no CPU fallback: if the library or a GPU is
missing the calls raise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libslepc_b200.so")

# EPSWhich
LARGEST_MAGNITUDE, SMALLEST_MAGNITUDE, LARGEST_REAL, SMALLEST_REAL = 1, 2, 3, 4
# EPSConvergedReason
CONVERGED_TOL, CONVERGED_ITERATING, DIVERGED_ITS, DIVERGED_BREAKDOWN = 1, 0, -1, -2
# EPSErrorType / SVDErrorType
ERROR_ABSOLUTE, ERROR_RELATIVE, ERROR_NORM = 0, 1, 2
# MatScalar storage of matrix values
SCALAR_F64, SCALAR_F32 = 0, 1

_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "LAPACK error", 4: "invalid inner product",
           5: "breakdown", 6: "out of device memory", 7: "wrong call order", 8: "device-side error",
           9: "floating-point error", 10: "file error"}

# PETSc binary files
MAT_FILE_CLASSID, VEC_FILE_CLASSID = 1211216, 1211214
FILE_MODE_READ, FILE_MODE_WRITE, FILE_MODE_APPEND = 0, 1, 2
MAT_OPERATOR = -1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_ll = ctypes.c_longlong
_lib = None


class B200Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"slepc_b200: {_STATUS.get(status, status)}: {msg}")
        self.status = status


class EPSStats(ctypes.Structure):
    _fields_ = [("lanczos_steps", ctypes.c_int64), ("gs_passes", ctypes.c_int64), ("restarts", ctypes.c_int64),
                ("kernel_launches", ctypes.c_int64), ("ms_spmv", ctypes.c_double), ("ms_orth", ctypes.c_double),
                ("ms_restart", ctypes.c_double), ("ms_total", ctypes.c_double), ("gs_bytes", ctypes.c_int64),
                ("column_visits", ctypes.c_int64), ("filter_sweeps", ctypes.c_int64),
                ("filter_degree", ctypes.c_int64), ("block_size", ctypes.c_int64),
                ("phase1_restarts", ctypes.c_int64), ("ms_phase1", ctypes.c_double), ("ms_phase2", ctypes.c_double),
                ("spmm_columns", ctypes.c_int64)]


_SIGS = {
    "b200_version": (ctypes.c_char_p, []),
    "b200_last_error": (ctypes.c_char_p, []),
    "b200_kernel_launch_count": (ctypes.c_uint64, []),
    "b200_mat_create_csr": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp, _vp, _vp]),
    "b200_mat_create_csr_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "b200_mat_mult": (ctypes.c_int, [_vp, _vp, _vp]),
    "b200_mat_get_size": (ctypes.c_int, [_vp, _ip, ctypes.POINTER(ctypes.c_int64)]),
    "b200_mat_get_lanes": (ctypes.c_int, [_vp, _ip]),
    "b200_mat_set_spmv_schedule": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_mat_destroy": (ctypes.c_int, [_vp]),
    "b200_mat_create_aij": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int64, _ip, _ip, _vp, ctypes.c_int,
                                           _vp, _vp]),
    "b200_mat_create_cross": (ctypes.c_int, [_vp, _vp]),
    "b200_mat_mult_transpose": (ctypes.c_int, [_vp, _vp, _vp]),
    "b200_mat_get_sizes": (ctypes.c_int, [_vp, _ip, _ip]),
    "b200_mat_norm_inf": (ctypes.c_int, [_vp, _dp]),
    "b200_eps_set_type": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_monitor_set": (ctypes.c_int, [_vp, _vp, _vp]),
    "b200_eps_monitor_cancel": (ctypes.c_int, [_vp]),
    "b200_eps_monitor_jsonl": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "b200_eps_krylovschur_set_locking": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_krylovschur_get_locking": (ctypes.c_int, [_vp, _ip]),
    "b200_bv_gram_schmidt": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _dp, _dp]),
    "b200_bv_resize": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "b200_bv_copy": (ctypes.c_int, [_vp, _vp]),
    "b200_bv_normalize": (ctypes.c_int, [_vp, _dp]),
    "b200_bv_mult_inplace_trans": (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_rowblock_gram": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp]),
    "b200_eps_solve_csr_host_ex": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp, _dp, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _ip, _vp]),
    "b200_rowblock_spmm": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, _vp]),
    "b200_tc_sgemm_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                           _vp, _ll, _ll, _ll, _vp, _ll, _ll, _ll, ctypes.c_float, _vp, _ll, _ll, _ll,
                                           ctypes.c_int, _vp, ctypes.c_size_t, _vp, _vp]),
    "b200_tc_sgemm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp,
                                     _ll, _ll, _ll, _vp, _ll, _ll, _ll, ctypes.c_float, _vp, _ll, _ll, _ll,
                                     ctypes.c_int, ctypes.c_int, _vp]),
    "b200_eps_set_mixed_options": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int]),
    "b200_eps_lobpcg_set_block_size": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_lobpcg_set_restart": (ctypes.c_int, [_vp, ctypes.c_double]),
    "b200_eps_lobpcg_set_locking": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_set_preconditioner": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_set_bv_orthog_block": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_set_initial_space_block": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_viewer_binary_open": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _vp]),
    "b200_viewer_destroy": (ctypes.c_int, [_vp]),
    "b200_viewer_peek": (ctypes.c_int, [_vp, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_int64)]),
    "b200_mat_read_csr": (ctypes.c_int, [_vp, _ip, _ip, _dp]),
    "b200_mat_write_csr": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp]),
    "b200_vec_read": (ctypes.c_int, [_vp, ctypes.c_int, _ip, _dp]),
    "b200_vec_write": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_mat_load": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "b200_mat_view": (ctypes.c_int, [_vp, _vp]),
    "b200_batch_create": (ctypes.c_int, [ctypes.c_int, _ip, _ip, _ip, _dp, _vp, _vp]),
    "b200_neural_op_create": (ctypes.c_int, [ctypes.c_int] * 6 + [_vp, _vp]),
    "b200_neural_op_destroy": (ctypes.c_int, [_vp]),
    "b200_neural_op_num_params": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "b200_neural_op_set_params": (ctypes.c_int, [_vp, _vp]),
    "b200_neural_op_get_params": (ctypes.c_int, [_vp, _vp]),
    "b200_neural_op_forward": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    "b200_neural_op_loss": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(ctypes.c_float)]),
    "b200_neural_op_loss_grad": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(ctypes.c_float), _vp]),
    "b200_neural_op_train_step": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_float,
                                                 ctypes.POINTER(ctypes.c_float)]),
    "b200_batch_destroy": (ctypes.c_int, [_vp]),
    "b200_batch_set_dimensions": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_batch_set_tolerances": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int]),
    "b200_batch_set_which_eigenpairs": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_batch_set_initial_vectors": (ctypes.c_int, [_vp, _dp]),
    "b200_batch_set_threads": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_batch_autotune": (ctypes.c_int, [_vp, _ip]),
    "b200_batch_solve": (ctypes.c_int, [_vp]),
    "b200_batch_get_solution": (ctypes.c_int, [_vp, ctypes.c_int, _ip, _ip, _ip, _ip, _dp, _dp]),
    "b200_batch_get_eigenvector": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp]),
    "b200_batch_get_all": (ctypes.c_int, [_vp, _dp, _ip, ctypes.POINTER(ctypes.c_float)]),
    "b200_batch_get_bytes": (ctypes.c_int, [_vp, _dp]),
    "b200_batch_set_precision": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "b200_batch_get_phase1": (ctypes.c_int, [_vp, _vp, _dp]),
    "b200_svd_create": (ctypes.c_int, [_vp, _vp]),
    "b200_svd_destroy": (ctypes.c_int, [_vp]),
    "b200_svd_set_operator": (ctypes.c_int, [_vp, _vp]),
    "b200_svd_set_dimensions": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_svd_set_tolerances": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int]),
    "b200_svd_set_which_singular_triplets": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_svd_set_initial_space": (ctypes.c_int, [_vp, _dp]),
    "b200_svd_set_timing": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_svd_solve": (ctypes.c_int, [_vp]),
    "b200_svd_get_converged": (ctypes.c_int, [_vp, _ip]),
    "b200_svd_get_iteration_number": (ctypes.c_int, [_vp, _ip]),
    "b200_svd_get_converged_reason": (ctypes.c_int, [_vp, _ip]),
    "b200_svd_get_singular_triplet": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _dp]),
    "b200_svd_get_singular_vectors_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                                            ctypes.POINTER(ctypes.c_void_p)]),
    "b200_svd_compute_error": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp]),
    "b200_svd_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(EPSStats)]),
    "b200_svd_solve_aij_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int64, _ip, _ip, _vp,
                                               ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_int, _dp, _dp, _dp, _dp, _ip, _vp]),
    "b200_csr_spmv": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "b200_bv_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "b200_bv_destroy": (ctypes.c_int, [_vp]),
    "b200_bv_get_sizes": (ctypes.c_int, [_vp, _ip, _ip, _ip]),
    "b200_bv_get_array": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_void_p)]),
    "b200_bv_set_active_columns": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "b200_bv_get_active_columns": (ctypes.c_int, [_vp, _ip, _ip]),
    "b200_bv_set_orthog_eta": (ctypes.c_int, [_vp, ctypes.c_double]),
    "b200_bv_set_orthog_block": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_bv_get_orthog_block": (ctypes.c_int, [_vp, _ip]),
    "b200_bv_set_column": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_bv_get_column": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_bv_copy_vec": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "b200_bv_insert_vec": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "b200_bv_orthogonalize_column": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _ip]),
    "b200_bv_orthonormalize_column": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _ip]),
    "b200_bv_orthogonalize_vec": (ctypes.c_int, [_vp, _vp, _dp, _dp, _ip]),
    "b200_bv_orthogonalize": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "b200_orthogonalize_column_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                                         ctypes.c_int, _vp, _dp, _ip, _vp]),
    "b200_bv_mult_inplace": (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_bv_mult_inplace_device": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_bv_mult": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vp, _dp, ctypes.c_int]),
    "b200_bv_mult_vec": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vp, _dp]),
    "b200_bv_dot": (ctypes.c_int, [_vp, _vp, _dp, ctypes.c_int]),
    "b200_bv_dot_vec": (ctypes.c_int, [_vp, _vp, _dp]),
    "b200_bv_scale_column": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "b200_bv_norm_column": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_bv_norm": (ctypes.c_int, [_vp, _dp]),
    "b200_bv_copy_column": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "b200_bv_mat_mult_column": (ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    "b200_bv_mat_mult": (ctypes.c_int, [_vp, _vp, _vp]),
    "b200_bv_mat_lanczos": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _ip, _dp, _dp, _dp, _ip]),
    "b200_eps_create": (ctypes.c_int, [_vp, _vp]),
    "b200_eps_destroy": (ctypes.c_int, [_vp]),
    "b200_eps_set_operators": (ctypes.c_int, [_vp, _vp]),
    "b200_eps_set_dimensions": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "b200_eps_set_tolerances": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int]),
    "b200_eps_set_which_eigenpairs": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_krylovschur_set_restart": (ctypes.c_int, [_vp, ctypes.c_double]),
    "b200_eps_set_initial_space": (ctypes.c_int, [_vp, _dp]),
    "b200_eps_set_initial_space_device": (ctypes.c_int, [_vp, _vp]),
    "b200_eps_set_max_restarts": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_set_timing": (ctypes.c_int, [_vp, ctypes.c_int]),
    "b200_eps_solve": (ctypes.c_int, [_vp]),
    "b200_eps_get_converged": (ctypes.c_int, [_vp, _ip]),
    "b200_eps_get_iteration_number": (ctypes.c_int, [_vp, _ip]),
    "b200_eps_get_converged_reason": (ctypes.c_int, [_vp, _ip]),
    "b200_eps_get_eigenpair": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp]),
    "b200_eps_get_eigenvector_device": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "b200_eps_get_error_estimate": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "b200_eps_compute_error": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp]),
    "b200_eps_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(EPSStats)]),
    "b200_eps_solve_csr_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _ip, _ip, _dp, _dp, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                               ctypes.c_int, _dp, _dp, _dp, _ip, _vp]),
}


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise B200Error(2, f"{LIB_PATH} is missing: build it with `python slepc_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS.keys())


def _check(status):
    if status != 0:
        raise B200Error(status, lib().b200_last_error().decode())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def kernel_launch_count():
    return int(lib().b200_kernel_launch_count())


class Viewer:
    """PETSc binary file (PetscViewerBinary) holding Mat and Vec objects in sequence."""

    class Mode:
        READ, WRITE, APPEND = 0, 1, 2

    def __init__(self):
        self.handle = ctypes.c_void_p()

    def createBinary(self, name, mode=0):
        _check(lib().b200_viewer_binary_open(os.fsencode(name), mode, ctypes.byref(self.handle)))
        return self

    def peek(self):
        """(classid, m, n, nnz) of the next object, without consuming it."""
        c, m, n, z = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        _check(lib().b200_viewer_peek(self.handle, ctypes.byref(c), ctypes.byref(m), ctypes.byref(n),
                                      ctypes.byref(z)))
        return c.value, m.value, n.value, z.value

    def readCSR(self):
        """The next Mat as host arrays (rowptr, colind, vals) and its shape."""
        _, m, n, nnz = self.peek()
        rowptr = np.zeros(m + 1, dtype=np.int32)
        colind = np.zeros(max(nnz, 1), dtype=np.int32)
        vals = np.zeros(max(nnz, 1))
        _check(lib().b200_mat_read_csr(self.handle, _i(rowptr), _i(colind), _d(vals)))
        return (rowptr, colind[:nnz], vals[:nnz]), (m, n)

    def writeCSR(self, csr, shape):
        rowptr = np.ascontiguousarray(csr[0], dtype=np.int32)
        colind = np.ascontiguousarray(csr[1], dtype=np.int32)
        vals = np.ascontiguousarray(csr[2], dtype=np.float64)
        _check(lib().b200_mat_write_csr(self.handle, shape[0], shape[1], int(rowptr[-1]), _i(rowptr), _i(colind),
                                        _d(vals)))

    def readVec(self):
        _, n, _, _ = self.peek()
        x = np.zeros(max(n, 1))
        got = ctypes.c_int()
        _check(lib().b200_vec_read(self.handle, len(x), ctypes.byref(got), _d(x)))
        return x[:got.value]

    def writeVec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        _check(lib().b200_vec_write(self.handle, len(x), _d(x)))

    def destroy(self):
        if self.handle:
            _check(lib().b200_viewer_destroy(self.handle))
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Mat:
    """CSR matrix resident in HBM (the new Mat SpMV type), or the cross shell A^T A."""

    def __init__(self):
        self.handle = ctypes.c_void_p()
        self.m = 0
        self.n = 0
        self.nnz = 0
        self._base = None

    def createAIJ(self, csr, size=None, dtype=None, stream=None):
        """Square FP64 CSR (size None, dtype None), or a general m x n matrix
        (size=(m, n)) with values stored as float64 or float32 (dtype); the
        general form also keeps the explicit transpose in HBM."""
        rowptr, colind, vals = csr
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        colind = np.ascontiguousarray(colind, dtype=np.int32)
        m = len(rowptr) - 1
        nnz = int(rowptr[-1])
        if size is None and dtype is None:
            vals = np.ascontiguousarray(vals, dtype=np.float64)
            _check(lib().b200_mat_create_csr(m, nnz, _i(rowptr), _i(colind), _d(vals), stream,
                                             ctypes.byref(self.handle)))
            self.m = self.n = m
        else:
            m, n = size if size is not None else (m, m)
            dt = np.dtype(dtype or np.float64)
            if dt not in (np.dtype(np.float32), np.dtype(np.float64)):
                raise B200Error(1, "values must be float32 or float64")
            vals = np.ascontiguousarray(vals, dtype=dt)
            st = SCALAR_F32 if dt == np.float32 else SCALAR_F64
            _check(lib().b200_mat_create_aij(m, n, nnz, _i(rowptr), _i(colind), vals.ctypes.data, st, stream,
                                             ctypes.byref(self.handle)))
            self.m, self.n = m, n
        self.nnz = nnz
        return self

    def load(self, viewer, storage=MAT_OPERATOR, stream=None):
        """MatLoad: the next Mat of a PETSc binary file, as a square operator
        (MAT_OPERATOR) or a general matrix stored SCALAR_F64 / SCALAR_F32."""
        _, m, n, nnz = viewer.peek()
        _check(lib().b200_mat_load(viewer.handle, storage, stream, ctypes.byref(self.handle)))
        self.m, self.n, self.nnz = m, n, nnz
        return self

    def view(self, viewer):
        """MatView to a PETSc binary file."""
        _check(lib().b200_mat_view(self.handle, viewer.handle))

    def createCross(self, A):
        """The shell A^T A (MatMult_Cross); A must outlive it."""
        _check(lib().b200_mat_create_cross(A.handle, ctypes.byref(self.handle)))
        self.m = self.n = A.n
        self.nnz = A.nnz
        self._base = A
        return self

    def getSizes(self):
        m, n = ctypes.c_int(), ctypes.c_int()
        _check(lib().b200_mat_get_sizes(self.handle, ctypes.byref(m), ctypes.byref(n)))
        return m.value, n.value

    def multTranspose(self, x_ptr, y_ptr):
        _check(lib().b200_mat_mult_transpose(self.handle, x_ptr, y_ptr))

    def norm(self):
        """MatNorm(NORM_INFINITY)."""
        v = ctypes.c_double()
        _check(lib().b200_mat_norm_inf(self.handle, ctypes.byref(v)))
        return v.value

    def createAIJDevice(self, n, nnz, rowptr_ptr, colind_ptr, vals_ptr, stream=None):
        _check(lib().b200_mat_create_csr_device(n, nnz, rowptr_ptr, colind_ptr, vals_ptr, stream,
                                                ctypes.byref(self.handle)))
        self.n, self.nnz = n, nnz
        return self

    def mult(self, x_ptr, y_ptr):
        _check(lib().b200_mat_mult(self.handle, x_ptr, y_ptr))

    ROWBLOCK, WARPTILE, PIPELINED, SELL = 0, 1, 2, 3

    def setSpMVSchedule(self, schedule):
        _check(lib().b200_mat_set_spmv_schedule(self.handle, schedule))

    def getLanes(self):
        v = ctypes.c_int()
        _check(lib().b200_mat_get_lanes(self.handle, ctypes.byref(v)))
        return v.value

    def destroy(self):
        if self.handle:
            lib().b200_mat_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class BV:
    """Column-major basis of vectors resident in HBM (the new BV type)."""

    class OrthogBlockType:
        """BVOrthogBlockType (include/slepcbv.h:84-88); TSQR and TSQRCHOL are the Householder QR of
        the active columns on the device (one process's geqrf + orgqr, R with LAPACK's signs)."""
        GS, CHOL, TSQR, TSQRCHOL, SVQB = 0, 1, 2, 3, 4

    def __init__(self):
        self.handle = ctypes.c_void_p()

    def create(self, n, m, stream=None):
        _check(lib().b200_bv_create(n, m, stream, ctypes.byref(self.handle)))
        return self

    def getSizes(self):
        n, m, ld = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().b200_bv_get_sizes(self.handle, ctypes.byref(n), ctypes.byref(m), ctypes.byref(ld)))
        return n.value, m.value, ld.value

    def getArrayPointer(self):
        p = ctypes.c_void_p()
        _check(lib().b200_bv_get_array(self.handle, ctypes.byref(p)))
        return p.value

    def setActiveColumns(self, l, k):
        _check(lib().b200_bv_set_active_columns(self.handle, l, k))

    def getActiveColumns(self):
        l, k = ctypes.c_int(), ctypes.c_int()
        _check(lib().b200_bv_get_active_columns(self.handle, ctypes.byref(l), ctypes.byref(k)))
        return l.value, k.value

    def setOrthogonalizationEta(self, eta):
        _check(lib().b200_bv_set_orthog_eta(self.handle, eta))

    def setOrthogonalizationBlock(self, block):
        """BVSetOrthogonalization's block type (BV.OrthogBlockType), the method of orthogonalize()."""
        _check(lib().b200_bv_set_orthog_block(self.handle, block))

    def getOrthogonalizationBlock(self):
        t = ctypes.c_int()
        _check(lib().b200_bv_get_orthog_block(self.handle, ctypes.byref(t)))
        return t.value

    def setColumn(self, j, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        _check(lib().b200_bv_set_column(self.handle, j, _d(x)))

    def getColumn(self, j):
        n = self.getSizes()[0]
        x = np.empty(n)
        _check(lib().b200_bv_get_column(self.handle, j, _d(x)))
        return x

    def setColumns(self, X):
        for j in range(X.shape[1]):
            self.setColumn(j, X[:, j])

    def getColumns(self, k=None):
        n, m, _ = self.getSizes()
        k = m if k is None else k
        return np.stack([self.getColumn(j) for j in range(k)], axis=1)

    def orthogonalizeColumn(self, j):
        """BVOrthogonalizeColumn: returns (H[0..j] with the norm last, norm, lindep)."""
        H = np.zeros(j + 1)
        nrm, lnd = ctypes.c_double(), ctypes.c_int()
        _check(lib().b200_bv_orthogonalize_column(self.handle, j, _d(H), ctypes.byref(nrm), ctypes.byref(lnd)))
        return H, nrm.value, bool(lnd.value)

    def orthonormalizeColumn(self, j):
        nrm, lnd = ctypes.c_double(), ctypes.c_int()
        _check(lib().b200_bv_orthonormalize_column(self.handle, j, ctypes.byref(nrm), ctypes.byref(lnd)))
        return nrm.value, bool(lnd.value)

    def orthogonalizeVec(self, v_ptr, k):
        H = np.zeros(max(k, 1))
        nrm, lnd = ctypes.c_double(), ctypes.c_int()
        _check(lib().b200_bv_orthogonalize_vec(self.handle, v_ptr, _d(H), ctypes.byref(nrm), ctypes.byref(lnd)))
        return H[:k], nrm.value, bool(lnd.value)

    def gramSchmidt(self, j, v_ptr=None, h_ptr=None, c_ptr=None, norms=True):
        """One classical Gram-Schmidt pass (the BV gramschmidt op, b200_bv_gram_schmidt): returns
        (onorm, norm) when norms is set (a synchronisation), else None."""
        if not norms:
            _check(lib().b200_bv_gram_schmidt(self.handle, j, v_ptr, h_ptr, c_ptr, None, None))
            return None
        on, nr = ctypes.c_double(), ctypes.c_double()
        _check(lib().b200_bv_gram_schmidt(self.handle, j, v_ptr, h_ptr, c_ptr, ctypes.byref(on), ctypes.byref(nr)))
        return on.value, nr.value

    def resize(self, m, copy=True):
        _check(lib().b200_bv_resize(self.handle, m, 1 if copy else 0))

    def copy(self, Y):
        """BVCopy: the active columns of this BV into Y from Y's leading column l."""
        _check(lib().b200_bv_copy(self.handle, Y.handle))

    def normalize(self):
        """BVNormalize (real): unit 2-norm active columns; returns their previous norms."""
        l, k = self.getActiveColumns()
        nrm = np.zeros(max(k - l, 1))
        _check(lib().b200_bv_normalize(self.handle, _d(nrm)))
        return nrm[: k - l]

    def multInPlaceTranspose(self, Q, s, e):
        """BVMultInPlaceHermitianTranspose (real): V(:,s:e) = V Q(s:e,:)^T."""
        Q = np.asfortranarray(Q, dtype=np.float64)
        _check(lib().b200_bv_mult_inplace_trans(self.handle, _d(Q), Q.shape[0], s, e))

    def orthogonalize(self, k):
        R = np.zeros((k, k), order="F")
        _check(lib().b200_bv_orthogonalize(self.handle, _d(R), k))
        return R

    def multInPlace(self, Q, s, e):
        Q = np.asfortranarray(Q, dtype=np.float64)
        _check(lib().b200_bv_mult_inplace(self.handle, _d(Q), Q.shape[0], s, e))

    def mult(self, alpha, beta, X, Q):
        Q = np.asfortranarray(Q, dtype=np.float64)
        _check(lib().b200_bv_mult(self.handle, alpha, beta, X.handle, _d(Q), Q.shape[0]))

    def multVec(self, alpha, beta, y_ptr, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        _check(lib().b200_bv_mult_vec(self.handle, alpha, beta, y_ptr, _d(q)))

    def dot(self, Y):
        """BVDot: M = Y^T X over the active columns (M is Y.k x X.k)."""
        _, kx = self.getActiveColumns()
        _, ky = Y.getActiveColumns()
        M = np.zeros((max(ky, 1), max(kx, 1)), order="F")
        _check(lib().b200_bv_dot(self.handle, Y.handle, _d(M), max(ky, 1)))
        return M[:ky, :kx]

    def dotVec(self, y_ptr, k):
        q = np.zeros(max(k, 1))
        _check(lib().b200_bv_dot_vec(self.handle, y_ptr, _d(q)))
        return q[:k]

    def scaleColumn(self, j, alpha):
        _check(lib().b200_bv_scale_column(self.handle, j, alpha))

    def scale(self, alpha):
        _check(lib().b200_bv_scale_column(self.handle, -1, alpha))

    def normColumn(self, j):
        v = ctypes.c_double()
        _check(lib().b200_bv_norm_column(self.handle, j, ctypes.byref(v)))
        return v.value

    def norm(self):
        v = ctypes.c_double()
        _check(lib().b200_bv_norm(self.handle, ctypes.byref(v)))
        return v.value

    def copyColumn(self, j, i):
        _check(lib().b200_bv_copy_column(self.handle, j, i))

    def matMultColumn(self, A, j):
        _check(lib().b200_bv_mat_mult_column(self.handle, A.handle, j))

    def matMult(self, A, Y):
        """BVMatMult: Y(:, Y.l+j) = A V(:, V.l+j) over the active columns."""
        _check(lib().b200_bv_mat_mult(self.handle, A.handle, Y.handle))

    def matLanczos(self, A, k, m):
        """BVMatLanczos: returns (alpha, beta_vec, m, beta, breakdown)."""
        mm = ctypes.c_int(m)
        alpha, betav = np.zeros(m + 1), np.zeros(m + 1)
        beta, bd = ctypes.c_double(), ctypes.c_int()
        _check(lib().b200_bv_mat_lanczos(self.handle, A.handle, k, ctypes.byref(mm), _d(alpha), _d(betav),
                                         ctypes.byref(beta), ctypes.byref(bd)))
        return alpha, betav, mm.value, beta.value, bool(bd.value)

    def destroy(self):
        if self.handle:
            lib().b200_bv_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class EPS:
    """Hermitian Krylov-Schur eigensolver (EPSKRYLOVSCHUR with EPS_HEP)."""

    class Which:
        LARGEST_MAGNITUDE, SMALLEST_MAGNITUDE, LARGEST_REAL, SMALLEST_REAL = 1, 2, 3, 4

    class ProblemType:
        HEP = 1

    class Type:
        KRYLOVSCHUR, LOBPCG = 0, 1

    class Precision:
        FP64 = 0
        MIXED = 1

    class PCType:
        NONE, JACOBI = 0, 1

    def __init__(self):
        self.handle = ctypes.c_void_p()
        self._A = None

    def create(self, stream=None):
        _check(lib().b200_eps_create(stream, ctypes.byref(self.handle)))
        return self

    def setOperators(self, A, B=None):
        if B is not None:
            raise B200Error(1, "only standard problems (B = None) are supported")
        self._A = A
        _check(lib().b200_eps_set_operators(self.handle, A.handle))

    def setProblemType(self, ptype):
        if ptype != EPS.ProblemType.HEP:
            raise B200Error(1, "only EPS_HEP is supported")

    def setDimensions(self, nev=1, ncv=0, mpd=0):
        _check(lib().b200_eps_set_dimensions(self.handle, nev, ncv or 0, mpd or 0))

    def setTolerances(self, tol=0.0, max_it=0):
        _check(lib().b200_eps_set_tolerances(self.handle, tol or 0.0, max_it or 0))

    def setWhichEigenpairs(self, which):
        _check(lib().b200_eps_set_which_eigenpairs(self.handle, which))

    def setKrylovSchurRestart(self, keep):
        _check(lib().b200_eps_krylovschur_set_restart(self.handle, keep))

    def setInitialSpace(self, v0):
        """One vector (length n) or a block (n x k array, columns are the vectors)."""
        v0 = np.asarray(v0, dtype=np.float64)
        if v0.ndim == 2:
            X = np.asfortranarray(v0)
            _check(lib().b200_eps_set_initial_space_block(self.handle, X.shape[1], _d(X)))
            return
        v0 = np.ascontiguousarray(v0)
        _check(lib().b200_eps_set_initial_space(self.handle, _d(v0)))

    def setType(self, t):
        _check(lib().b200_eps_set_type(self.handle, t))

    def setLOBPCGBlockSize(self, bs):
        _check(lib().b200_eps_lobpcg_set_block_size(self.handle, bs))

    def setLOBPCGRestart(self, restart):
        _check(lib().b200_eps_lobpcg_set_restart(self.handle, restart))

    def setLOBPCGLocking(self, lock):
        _check(lib().b200_eps_lobpcg_set_locking(self.handle, 1 if lock else 0))

    def setPreconditioner(self, pc):
        """STPRECOND with KSPPREONLY and PCNONE / PCJACOBI (EPS.PCType)."""
        _check(lib().b200_eps_set_preconditioner(self.handle, pc))

    def setBVOrthogonalizationBlock(self, block):
        """-bv_orthog_block: the BVOrthogBlockType (BV.OrthogBlockType) of the basis, which
        LOBPCG's blocks inherit."""
        _check(lib().b200_eps_set_bv_orthog_block(self.handle, block))

    def setPrecision(self, precision):
        """EPS.Precision.FP64 (default, the drop-in path) or EPS.Precision.MIXED: Krylov-Schur
        on an FP32 basis with FP32 matrix values to a loose tolerance, then FP64
        Chebyshev-filtered Rayleigh-Ritz refinement of the block of leading Ritz vectors."""
        _check(lib().b200_eps_set_precision(self.handle, precision))

    _MonitorFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                  ctypes.c_void_p)

    def setMonitor(self, fn):
        """EPSMonitorSet: fn(its, nconv, eigr, errest) is called once per outer iteration with numpy
        copies of the nest current values and estimates; a true return value aborts the solve."""
        def tramp(_eps, its, nconv, eigr, errest, nest, _ctx):
            try:
                r = fn(its, nconv, np.ctypeslib.as_array(eigr, (nest,)).copy(),
                       np.ctypeslib.as_array(errest, (nest,)).copy())
                return 1 if r else 0
            except Exception:
                return 1
        cb = self._MonitorFn(tramp)
        self._monitors = getattr(self, "_monitors", []) + [cb]  # keep the callbacks alive
        _check(lib().b200_eps_monitor_set(self.handle, ctypes.cast(cb, ctypes.c_void_p), None))

    def setMonitorJSONL(self, path):
        """The built-in monitor: one JSON line per outer iteration written to path."""
        _check(lib().b200_eps_monitor_jsonl(self.handle, os.fsencode(path)))

    def cancelMonitor(self):
        _check(lib().b200_eps_monitor_cancel(self.handle))
        self._monitors = []

    def setKrylovSchurLocking(self, lock):
        """EPSKrylovSchurSetLocking (the non-locking variant needs mpd = ncv)."""
        _check(lib().b200_eps_krylovschur_set_locking(self.handle, 1 if lock else 0))

    def getKrylovSchurLocking(self):
        v = ctypes.c_int()
        _check(lib().b200_eps_krylovschur_get_locking(self.handle, ctypes.byref(v)))
        return bool(v.value)

    def setMixedOptions(self, tol_low=0.0, degree=0, guard=-1, max_sweeps=0, fp64_gram=False):
        """Parameters of the mixed form (b200_eps_set_mixed_options); 0 (or -1 for guard) keeps the default."""
        _check(lib().b200_eps_set_mixed_options(self.handle, tol_low, degree, guard, max_sweeps,
                                                int(bool(fp64_gram))))

    def setInitialSpaceDevice(self, v0_ptr):
        _check(lib().b200_eps_set_initial_space_device(self.handle, v0_ptr))

    def setMaxRestarts(self, r):
        _check(lib().b200_eps_set_max_restarts(self.handle, r))

    def setTiming(self, on):
        _check(lib().b200_eps_set_timing(self.handle, 1 if on else 0))

    def solve(self):
        _check(lib().b200_eps_solve(self.handle))

    def getConverged(self):
        v = ctypes.c_int()
        _check(lib().b200_eps_get_converged(self.handle, ctypes.byref(v)))
        return v.value

    def getIterationNumber(self):
        v = ctypes.c_int()
        _check(lib().b200_eps_get_iteration_number(self.handle, ctypes.byref(v)))
        return v.value

    def getConvergedReason(self):
        v = ctypes.c_int()
        _check(lib().b200_eps_get_converged_reason(self.handle, ctypes.byref(v)))
        return v.value

    def getEigenpair(self, i, want_vector=True):
        lam = ctypes.c_double()
        x = np.empty(self._A.n) if want_vector else None
        _check(lib().b200_eps_get_eigenpair(self.handle, i, ctypes.byref(lam), _d(x) if want_vector else None))
        return (lam.value, x) if want_vector else lam.value

    def getEigenvalue(self, i):
        return self.getEigenpair(i, want_vector=False)

    def getEigenvectorPointer(self, i):
        p = ctypes.c_void_p()
        _check(lib().b200_eps_get_eigenvector_device(self.handle, i, ctypes.byref(p)))
        return p.value

    def getErrorEstimate(self, i):
        v = ctypes.c_double()
        _check(lib().b200_eps_get_error_estimate(self.handle, i, ctypes.byref(v)))
        return v.value

    def computeError(self, i, etype=ERROR_RELATIVE):
        v = ctypes.c_double()
        _check(lib().b200_eps_compute_error(self.handle, i, etype, ctypes.byref(v)))
        return v.value

    def getStats(self):
        s = EPSStats()
        _check(lib().b200_eps_get_stats(self.handle, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in EPSStats._fields_}

    def viewEigenvectors(self, viewer):
        """Append the converged eigenvectors to a PETSc binary file as Vecs, in order (a warm
        start for a later solve: read one back and pass it to setInitialSpace)."""
        for i in range(self.getConverged()):
            viewer.writeVec(self.getEigenpair(i)[1])

    def destroy(self):
        if self.handle:
            lib().b200_eps_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def orthogonalize_column_noalloc(n, ld, ncols, V_ptr, j, H_ptr, stream=None):
    """Allocation-free column orthogonalisation on caller-owned device memory
    (b200_orthogonalize_column_noalloc): returns (norm, lindep)."""
    nrm, lnd = ctypes.c_double(), ctypes.c_int()
    _check(lib().b200_orthogonalize_column_noalloc(n, ld, ncols, V_ptr, j, H_ptr, ctypes.byref(nrm),
                                                   ctypes.byref(lnd), stream))
    return nrm.value, bool(lnd.value)


def rowblock_gram(n, bp, X_ptr, Y_ptr=None, tensor_cores=True, G_ptr=None, stream=None):
    """G = X^T Y (bp x bp, FP64, row-major) of row-major FP32 device blocks (b200_rowblock_gram):
    on the tensor cores (TF32 inputs, FP32 accumulation) or in FP64 on the CUDA cores."""
    _check(lib().b200_rowblock_gram(n, bp, X_ptr, Y_ptr, 1 if tensor_cores else 0, G_ptr, stream))


def rowblock_spmm(A, bp, X_ptr, Y_ptr, Z_ptr=None, alpha=1.0, shift=0.0, beta=0.0, x32=True, stream=None):
    """Y = alpha (A X - shift X) - beta Z on row-major device blocks (b200_rowblock_spmm); A a Mat
    created from a square CSR."""
    _check(lib().b200_rowblock_spmm(A.handle, bp, 1 if x32 else 0, X_ptr, Z_ptr, Y_ptr, alpha, shift, beta, stream))


def tc_sgemm(batch, m, n, k, alpha, A, B, beta, C, split=False, sum_batch=False, stream=None):
    """C[z] = alpha A[z] B[z] + beta C[z] on the tensor cores (b200_tc_sgemm).  A, B and C are
    (ptr, rs, cs, bs) device views of FP32 matrices: element (i, j) of matrix z at
    ptr + z*bs + i*rs + j*cs (elements)."""
    _check(lib().b200_tc_sgemm(batch, m, n, k, alpha, *A, *B, beta, *C, 1 if split else 0, 1 if sum_batch else 0,
                               stream))


def tc_sgemm_async(batch, m, n, k, alpha, A, B, beta, C, ws=None, ws_floats=0, err=None, sum_batch=False,
                   stream=None):
    """b200_tc_sgemm_async: the same product queued without allocation or synchronisation; ws (device
    pointer, ws_floats floats) the split-depth workspace, err a device int for the error bits."""
    _check(lib().b200_tc_sgemm_async(batch, m, n, k, alpha, *A, *B, beta, *C, 1 if sum_batch else 0, ws, ws_floats,
                                     err, stream))


def solve_csr_host(csr, v0, nev, ncv, tol=1e-8, which=LARGEST_MAGNITUDE, mpd=0, max_it=0, want_vectors=True,
                   stream=None, out=None, precision=0):
    """One call from host CSR arrays to host eigenpairs (b200_eps_solve_csr_host_ex).  out: an optional
    C-contiguous float64 array of shape (ncv + 1, n), (max(ncv + 1, 128), n) for the mixed form, that
    receives the eigenvectors (row i = vector i), for callers that keep a reused (for instance
    page-locked) output buffer.  precision: EPS.Precision.FP64 (0) or MIXED (1)."""
    rowptr, colind, vals = (np.ascontiguousarray(csr[0], dtype=np.int32), np.ascontiguousarray(csr[1], dtype=np.int32),
                            np.ascontiguousarray(csr[2], dtype=np.float64))
    n = len(rowptr) - 1
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    rows = ncv + 1 if not precision else max(ncv + 1, 128)  # the mixed form returns up to its block size
    evals = np.zeros(rows)
    errest = np.zeros(rows)
    # np.empty: only the rows the library writes (nconv of them) are ever touched
    if want_vectors and out is not None:
        if out.shape != (rows, n) or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
            raise B200Error(1, f"out must be a C-contiguous float64 array of shape ({rows}, n)")
        X = out
    else:
        X = np.empty((rows, n)) if want_vectors else None
    info = np.zeros(8, dtype=np.int32)
    _check(lib().b200_eps_solve_csr_host_ex(n, int(rowptr[-1]), _i(rowptr), _i(colind), _d(vals), _d(v0), nev, ncv,
                                            mpd, tol, max_it, which, int(precision), _d(evals),
                                            _d(X) if want_vectors else None, _d(errest), _i(info), stream))
    nconv = int(info[0])
    return {"evals": evals[:nconv].copy(), "X": X[:nconv].T if want_vectors else None,
            "errest": errest[:nconv].copy(), "nconv": nconv, "its": int(info[1]), "reason": int(info[2]),
            "lanczos_steps": int(info[3]), "restarts": int(info[4])}


class SVD:
    """SVD cross solver (SVDCROSS): Krylov-Schur on A^T A."""

    class Which:
        LARGEST, SMALLEST = 0, 1

    class ErrorType:
        ABSOLUTE, RELATIVE, NORM = 0, 1, 2

    def __init__(self):
        self.handle = ctypes.c_void_p()
        self._A = None

    def create(self, stream=None):
        _check(lib().b200_svd_create(stream, ctypes.byref(self.handle)))
        return self

    def setOperators(self, A, B=None):
        if B is not None:
            raise B200Error(1, "only standard problems (B = None) are supported")
        self._A = A
        _check(lib().b200_svd_set_operator(self.handle, A.handle))

    def setDimensions(self, nsv=1, ncv=0, mpd=0):
        _check(lib().b200_svd_set_dimensions(self.handle, nsv, ncv or 0, mpd or 0))

    def setTolerances(self, tol=0.0, max_it=0):
        _check(lib().b200_svd_set_tolerances(self.handle, tol or 0.0, max_it or 0))

    def setWhichSingularTriplets(self, which):
        _check(lib().b200_svd_set_which_singular_triplets(self.handle, which))

    def setInitialSpace(self, v0):
        v0 = np.ascontiguousarray(v0, dtype=np.float64)
        _check(lib().b200_svd_set_initial_space(self.handle, _d(v0)))

    def setTiming(self, on):
        _check(lib().b200_svd_set_timing(self.handle, 1 if on else 0))

    def solve(self):
        _check(lib().b200_svd_solve(self.handle))

    def getConverged(self):
        v = ctypes.c_int()
        _check(lib().b200_svd_get_converged(self.handle, ctypes.byref(v)))
        return v.value

    def getIterationNumber(self):
        v = ctypes.c_int()
        _check(lib().b200_svd_get_iteration_number(self.handle, ctypes.byref(v)))
        return v.value

    def getConvergedReason(self):
        v = ctypes.c_int()
        _check(lib().b200_svd_get_converged_reason(self.handle, ctypes.byref(v)))
        return v.value

    def getValue(self, i):
        s = ctypes.c_double()
        _check(lib().b200_svd_get_singular_triplet(self.handle, i, ctypes.byref(s), None, None))
        return s.value

    def getSingularTriplet(self, i):
        """(sigma, u, v) with u of length m and v of length n."""
        s = ctypes.c_double()
        u = np.empty(self._A.m)
        v = np.empty(self._A.n)
        _check(lib().b200_svd_get_singular_triplet(self.handle, i, ctypes.byref(s), _d(u), _d(v)))
        return s.value, u, v

    def getVectorPointers(self, i):
        u, v = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().b200_svd_get_singular_vectors_device(self.handle, i, ctypes.byref(u), ctypes.byref(v)))
        return u.value, v.value

    def computeError(self, i, etype=ERROR_RELATIVE):
        v = ctypes.c_double()
        _check(lib().b200_svd_compute_error(self.handle, i, etype, ctypes.byref(v)))
        return v.value

    def getStats(self):
        st = EPSStats()
        _check(lib().b200_svd_get_stats(self.handle, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in EPSStats._fields_}

    def destroy(self):
        if self.handle:
            lib().b200_svd_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def svd_solve_aij_host(csr, size, v0, nsv, ncv, tol=0.0, max_it=0, dtype=np.float64, want_vectors=True,
                       stream=None):
    """One call from host CSR arrays to host singular triplets (b200_svd_solve_aij_host)."""
    m, n = size
    rowptr = np.ascontiguousarray(csr[0], dtype=np.int32)
    colind = np.ascontiguousarray(csr[1], dtype=np.int32)
    dt = np.dtype(dtype)
    vals = np.ascontiguousarray(csr[2], dtype=dt)
    st = SCALAR_F32 if dt == np.float32 else SCALAR_F64
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    sig = np.zeros(ncv + 1)
    err = np.zeros(ncv + 1)
    U = np.empty((ncv + 1, m)) if want_vectors else None
    V = np.empty((ncv + 1, n)) if want_vectors else None
    info = np.zeros(8, dtype=np.int32)
    _check(lib().b200_svd_solve_aij_host(m, n, int(rowptr[-1]), _i(rowptr), _i(colind), vals.ctypes.data, st, _d(v0),
                                         nsv, ncv, tol, max_it, _d(sig), _d(U) if want_vectors else None,
                                         _d(V) if want_vectors else None, _d(err), _i(info), stream))
    k = int(info[0])
    return {"sigma": sig[:k].copy(), "U": U[:k].T if want_vectors else None,
            "V": V[:k].T if want_vectors else None, "rel_error": err[:k].copy(), "nconv": k,
            "its": int(info[1]), "reason": int(info[2]), "lanczos_steps": int(info[3]), "restarts": int(info[4])}


class NeuralOperator:
    """The neural-operator warm start (b200_neural_op_*): features and targets are CUDA float32
    tensors of shape (batch, 3, N*N) and (batch, nout, N*N); parameters are a flat float32 array."""

    def __init__(self):
        self.handle = ctypes.c_void_p()

    def create(self, N, width=32, modes=16, layers=4, hidden=64, nout=16, stream=None):
        _check(lib().b200_neural_op_create(N, width, modes, layers, hidden, nout, stream, ctypes.byref(self.handle)))
        self.dims = (N, width, modes, layers, hidden, nout)
        return self

    def destroy(self):
        if self.handle:
            _check(lib().b200_neural_op_destroy(self.handle))
            self.handle = ctypes.c_void_p()

    def numParams(self):
        n = ctypes.c_int64()
        _check(lib().b200_neural_op_num_params(self.handle, ctypes.byref(n)))
        return n.value

    def setParams(self, theta):
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        assert theta.size == self.numParams()
        _check(lib().b200_neural_op_set_params(self.handle, theta.ctypes.data))

    def getParams(self):
        out = np.empty(self.numParams(), dtype=np.float32)
        _check(lib().b200_neural_op_get_params(self.handle, out.ctypes.data))
        return out

    @staticmethod
    def _dense(t):
        """The kernels read dense (batch, channels, N*N) float32 device memory."""
        import torch

        if not t.is_cuda:
            raise B200Error(1, "neural-operator tensors must be on the GPU")
        return t.to(torch.float32).contiguous()

    def forward(self, features):
        import torch

        features = self._dense(features)
        N, _, _, _, _, K = self.dims
        out = torch.empty((features.shape[0], K, N * N), dtype=torch.float32, device=features.device)
        _check(lib().b200_neural_op_forward(self.handle, features.shape[0], features.data_ptr(), out.data_ptr()))
        return out

    def loss(self, features, targets):
        features, targets = self._dense(features), self._dense(targets)
        v = ctypes.c_float()
        _check(lib().b200_neural_op_loss(self.handle, features.shape[0], features.data_ptr(), targets.data_ptr(),
                                         ctypes.byref(v)))
        return v.value

    def lossGrad(self, features, targets):
        features, targets = self._dense(features), self._dense(targets)
        v = ctypes.c_float()
        g = np.empty(self.numParams(), dtype=np.float32)
        _check(lib().b200_neural_op_loss_grad(self.handle, features.shape[0], features.data_ptr(),
                                              targets.data_ptr(), ctypes.byref(v), g.ctypes.data))
        return v.value, g

    def trainStep(self, features, targets, lr):
        features, targets = self._dense(features), self._dense(targets)
        v = ctypes.c_float()
        _check(lib().b200_neural_op_train_step(self.handle, features.shape[0], features.data_ptr(),
                                               targets.data_ptr(), lr, ctypes.byref(v)))
        return v.value


class BatchEPS:
    """Many independent small Hermitian eigenproblems by Krylov-Schur in one persistent launch."""

    def __init__(self):
        self.handle = ctypes.c_void_p()
        self.ns = None
        self.ncv = 0

    def create(self, ns, rowptr, colind, vals, stream=None):
        """ns: problem sizes; rowptr: local row pointers one after another; colind/vals: nonzeros."""
        self.ns = np.ascontiguousarray(ns, dtype=np.int32)
        self._keep = (np.ascontiguousarray(rowptr, dtype=np.int32), np.ascontiguousarray(colind, dtype=np.int32),
                      np.ascontiguousarray(vals, dtype=np.float64))
        _check(lib().b200_batch_create(len(self.ns), _i(self.ns), _i(self._keep[0]), _i(self._keep[1]),
                                       _d(self._keep[2]), stream, ctypes.byref(self.handle)))
        self._keep = None
        return self

    def setDimensions(self, nev, ncv=0, mpd=0):
        _check(lib().b200_batch_set_dimensions(self.handle, nev, ncv, mpd))
        self.nev = nev
        self.ncv = ncv or max(2 * nev, nev + 15)

    def setTolerances(self, tol=0.0, max_it=0):
        _check(lib().b200_batch_set_tolerances(self.handle, tol, max_it))

    def setWhichEigenpairs(self, which):
        _check(lib().b200_batch_set_which_eigenpairs(self.handle, which))

    def setInitialVectors(self, v0):
        v0 = np.ascontiguousarray(v0, dtype=np.float64)
        _check(lib().b200_batch_set_initial_vectors(self.handle, _d(v0)))

    def setThreads(self, threads):
        _check(lib().b200_batch_set_threads(self.handle, threads))

    def autotune(self):
        t = ctypes.c_int()
        _check(lib().b200_batch_autotune(self.handle, ctypes.byref(t)))
        return t.value

    def solve(self):
        _check(lib().b200_batch_solve(self.handle))

    def getSolution(self, p):
        nconv, its, reason, steps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ev = np.zeros(max(self.ncv, 1))
        er = np.zeros(max(self.ncv, 1))
        _check(lib().b200_batch_get_solution(self.handle, p, ctypes.byref(nconv), ctypes.byref(its),
                                             ctypes.byref(reason), ctypes.byref(steps), _d(ev), _d(er)))
        k = nconv.value
        return {"nconv": k, "its": its.value, "reason": reason.value, "lanczos_steps": steps.value,
                "evals": ev[:k].copy(), "errest": er[:k].copy()}

    def getEigenvector(self, p, i):
        x = np.zeros(int(self.ns[p]))
        _check(lib().b200_batch_get_eigenvector(self.handle, p, i, _d(x)))
        return x

    def getAll(self):
        ev = np.zeros((len(self.ns), self.ncv))
        info = np.zeros((len(self.ns), 8), dtype=np.int32)
        ms = ctypes.c_float()
        _check(lib().b200_batch_get_all(self.handle, _d(ev), _i(info), ctypes.byref(ms)))
        return ev, info, ms.value

    def getBytes(self):
        """Algorithmic bytes moved by the last solve (for the HBM roofline)."""
        v = ctypes.c_double()
        _check(lib().b200_batch_get_bytes(self.handle, ctypes.byref(v)))
        return v.value

    def setPrecision(self, precision, tol_low=0.0):
        """EPS.Precision.FP64 (default) or EPS.Precision.MIXED: phase 1 on FP32 bases to tol_low, then
        the FP64 solve of every problem from the sum of its phase-1 Ritz vectors."""
        _check(lib().b200_batch_set_precision(self.handle, precision, tol_low))

    def getPhase1(self):
        """Phase-1 counters of the last mixed solve: (info (nprob x 8), algorithmic bytes)."""
        info = np.zeros((len(self.ns), 8), dtype=np.int32)
        v = ctypes.c_double()
        _check(lib().b200_batch_get_phase1(self.handle, info.ctypes.data, ctypes.byref(v)))
        return info, v.value

    def destroy(self):
        if self.handle:
            lib().b200_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
