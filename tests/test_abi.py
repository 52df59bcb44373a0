"""The C-ABI library loads and exports every entry point the headers declare (CPU only)."""
import ctypes
import glob
import os
import re

import pytest

from tests.conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(b200_[A-Za-z0-9_]+)\s*\(", txt, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "b200_eps_solve" in names and "b200_bv_orthogonalize_column" in names and "b200_mat_mult" in names
    assert len(names) >= 50


def test_library_exports_every_declared_symbol(b200):
    lib = ctypes.CDLL(b200.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_covers_header(b200):
    missing = sorted(set(declared_functions()) - set(b200.exported_symbols()))
    assert not missing, missing


def test_entry_points_reject_bad_arguments(b200):
    import numpy as np

    L = b200.lib()
    h = ctypes.c_void_p()
    # n <= 0
    assert L.b200_mat_create_csr(0, 0, None, None, None, None, ctypes.byref(h)) == 1
    # rowptr not ending at nnz
    rowptr = np.array([0, 1, 3], dtype=np.int32)
    colind = np.array([0, 1, 1], dtype=np.int32)
    vals = np.ones(3)
    rc = L.b200_mat_create_csr(2, 2, rowptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               colind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, ctypes.byref(h))
    assert rc == 1 and b"rowptr" in L.b200_last_error()
    # too many BV columns for the kernels
    assert L.b200_bv_create(100, 400, None, ctypes.byref(h)) == 1
    assert L.b200_eps_set_dimensions(None, 1, 0, 0) == 1
    # block orthogonalization type on missing objects
    assert L.b200_bv_set_orthog_block(None, 1) == 1
    assert L.b200_eps_set_bv_orthog_block(None, 4) == 1
    t = ctypes.c_int(-1)
    assert L.b200_bv_get_orthog_block(None, ctypes.byref(t)) == 1
    with pytest.raises(b200.B200Error):
        b200._check(1)
