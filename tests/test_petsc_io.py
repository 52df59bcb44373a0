"""PETSc binary Mat/Vec I/O (MatLoad/MatView, VecLoad/VecView format) against the two
binary files of SLEPc's ex31 tutorial (decoded into tests/golden/petsc_binary.json by
make_golden.py), plus the MatLoad -> EPSSolve path on the GPU."""
import json
import os
import struct

import numpy as np
import pytest

import slepc_b200 as S
from slepc_b200 import problems as P

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    with open(os.path.join(HERE, "golden", "petsc_binary.json")) as f:
        return json.load(f)["files"]


def _vec_bytes(vals):
    return struct.pack(">ii", 1211214, len(vals)) + struct.pack(">%dd" % len(vals), *vals)


def _mat_bytes(m, n, lens, cols, vals):
    return (struct.pack(">iiii", 1211216, m, n, len(cols)) + struct.pack(">%di" % m, *lens)
            + struct.pack(">%di" % len(cols), *cols) + struct.pack(">%dd" % len(vals), *vals))


def _fixture_objects():
    g = _golden()
    x = [float.fromhex(h) for h in g["X.bin"]["values_hex"]]
    y = g["Ybus.bin"]
    yv = [float.fromhex(h) for h in y["values_hex"]]
    return g, x, y, yv


def test_reads_the_reference_binary_files(tmp_path):
    g, x, y, yv = _fixture_objects()
    xb, yb = _vec_bytes(x), _mat_bytes(y["m"], y["n"], y["row_lengths"], y["colind"], yv)
    assert len(xb) == g["X.bin"]["bytes"] and len(yb) == g["Ybus.bin"]["bytes"]
    (tmp_path / "X.bin").write_bytes(xb)
    (tmp_path / "Ybus.bin").write_bytes(yb)
    with S.Viewer().createBinary(str(tmp_path / "X.bin")) as v:
        assert v.peek() == (S.VEC_FILE_CLASSID, 18, 1, 18)
        got = v.readVec()
    assert np.array_equal(got, np.array(x))
    with S.Viewer().createBinary(str(tmp_path / "Ybus.bin")) as v:
        assert v.peek() == (S.MAT_FILE_CLASSID, 18, 18, 108)
        (rowptr, colind, vals), shape = v.readCSR()
    assert shape == (18, 18)
    assert np.array_equal(np.diff(rowptr), y["row_lengths"])
    assert np.array_equal(colind, y["colind"]) and np.array_equal(vals, np.array(yv))


def test_writes_the_reference_bytes(tmp_path):
    g, x, y, yv = _fixture_objects()
    rowptr = np.concatenate([[0], np.cumsum(y["row_lengths"])]).astype(np.int32)
    with S.Viewer().createBinary(str(tmp_path / "out.bin"), S.FILE_MODE_WRITE) as v:
        v.writeVec(np.array(x))
        v.writeCSR((rowptr, np.array(y["colind"]), np.array(yv)), (y["m"], y["n"]))
    data = (tmp_path / "out.bin").read_bytes()
    assert data == _vec_bytes(x) + _mat_bytes(y["m"], y["n"], y["row_lengths"], y["colind"], yv)


def test_object_sequence_append_and_errors(tmp_path):
    f = str(tmp_path / "seq.bin")
    csr = P.laplacian_2d(5)
    with S.Viewer().createBinary(f, S.FILE_MODE_WRITE) as v:
        v.writeVec(np.arange(3.0))
    with S.Viewer().createBinary(f, S.FILE_MODE_APPEND) as v:
        v.writeCSR(csr, (25, 25))
        v.writeVec(np.array([]))
    with S.Viewer().createBinary(f) as v:
        assert np.array_equal(v.readVec(), [0.0, 1.0, 2.0])
        with pytest.raises(S.B200Error) as e:
            v.readVec()  # the next object is a Mat: nothing consumed
        assert e.value.status == 10
        (rp, ci, va), shape = v.readCSR()
        assert shape == (25, 25) and np.array_equal(rp, csr[0]) and np.array_equal(ci, csr[1])
        assert np.array_equal(va, csr[2])
        assert len(v.readVec()) == 0
        with pytest.raises(S.B200Error) as e:
            v.peek()
        assert e.value.status == 10
    # truncated and foreign files
    data = open(f, "rb").read()
    (tmp_path / "trunc.bin").write_bytes(data[:-5])
    with S.Viewer().createBinary(str(tmp_path / "trunc.bin")) as v:
        v.readVec()
        v.readCSR()
        with pytest.raises(S.B200Error):
            v.readVec()
    (tmp_path / "junk.bin").write_bytes(b"not a petsc file at all")
    with S.Viewer().createBinary(str(tmp_path / "junk.bin")) as v:
        with pytest.raises(S.B200Error):
            v.peek()
    with pytest.raises(S.B200Error):
        S.Viewer().createBinary(str(tmp_path / "missing" / "x.bin"))


@pytest.mark.gpu
def test_matload_then_solve_matches_direct_creation(tmp_path):
    csr = P.laplacian_2d(30, 31)
    n = len(csr[0]) - 1
    f = str(tmp_path / "lap.bin")
    with S.Viewer().createBinary(f, S.FILE_MODE_WRITE) as v:
        v.writeCSR(csr, (n, n))
    v0 = P.start_vector(n, 0)

    def solve(A):
        E = S.EPS().create()
        E.setOperators(A)
        E.setDimensions(6, 24)
        E.setTolerances(1e-10)
        E.setInitialSpace(v0)
        E.solve()
        return E, [E.getEigenpair(i) for i in range(E.getConverged())]

    with S.Viewer().createBinary(f) as v:
        A1 = S.Mat().load(v)
    E1, r1 = solve(A1)
    E2, r2 = solve(S.Mat().createAIJ(csr))
    assert len(r1) == len(r2) >= 6
    for (l1, x1), (l2, x2) in zip(r1, r2):
        assert l1 == l2 and np.array_equal(x1, x2)
    # warm start round trip: eigenvectors saved as Vecs, read back
    g = str(tmp_path / "evecs.bin")
    with S.Viewer().createBinary(g, S.FILE_MODE_WRITE) as v:
        E1.viewEigenvectors(v)
    with S.Viewer().createBinary(g) as v:
        back = [v.readVec() for _ in range(len(r1))]
    assert all(np.array_equal(b, x) for b, (_, x) in zip(back, r1))
    # MatView of a loaded matrix reproduces the file
    h = str(tmp_path / "again.bin")
    with S.Viewer().createBinary(h, S.FILE_MODE_WRITE) as v:
        A1.view(v)
    assert open(h, "rb").read() == open(f, "rb").read()


@pytest.mark.gpu
def test_matload_general_fp32_and_view(tmp_path):
    m, n = 700, 300
    rowptr, colind, vals = P.powerlaw_rect(m, n, 12, 1.8, 3)
    f = str(tmp_path / "rect.bin")
    with S.Viewer().createBinary(f, S.FILE_MODE_WRITE) as v:
        v.writeCSR((rowptr, colind, vals.astype(np.float64)), (m, n))
    with S.Viewer().createBinary(f) as v:
        A = S.Mat().load(v, S.SCALAR_F32)
    assert A.getSizes() == (m, n)
    g = str(tmp_path / "rect2.bin")
    with S.Viewer().createBinary(g, S.FILE_MODE_WRITE) as v:
        A.view(v)
    assert open(g, "rb").read() == open(f, "rb").read()
    with S.Viewer().createBinary(f) as v:
        with pytest.raises(S.B200Error):
            S.Mat().load(v, S.MAT_OPERATOR)  # not square
