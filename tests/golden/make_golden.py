"""Regenerate the golden fixtures in this folder from SLEPc's own test outputs.

Reads the reference's expected-output files (text) and the fixture formulas of
the corresponding test programs, and writes small JSON files that the tests
compare against.  Run it where the SLEPc source tree is available:

    python tests/golden/make_golden.py /path/to/slepc

The JSON files are committed; the tests never read the SLEPc tree.

Sources:
  src/eps/tutorials/output/ex2_1.out, ex2_1_alt.out   (ex2.c -n 72 -eps_nev 4 -eps_ncv 20)
  src/eps/tests/output/test2_1.out                     (test2.c, 1-D Laplacian n=30, locking 0 and 1)
  src/sys/classes/bv/tests/output/test2_1.out         (test2.c, n=20 k=8, CGS)
  src/sys/classes/ds/tests/output/test2_1.out         (test2.c, DSHEP n=12, ld=n+2)
  src/sys/classes/bv/tests/output/test1_1_bv_type-svec.out (test1.c, n=10 k=5 l=3, -verbose)
  src/sys/classes/bv/tests/output/test11_1.out, test11_6.out (test11.c, n=20 l=2 k=8, block types)
  src/eps/tutorials/X.bin, Ybus.bin                    (PETSc binary Vec and Mat read by ex31.c)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def ex2(root):
    out = {}
    for name in ("ex2_1.out", "ex2_1_alt.out"):
        txt = read(root, "src/eps/tutorials/output/" + name)
        m = re.search(r"N=(\d+) \((\d+)x(\d+) grid\)", txt)
        vals_line = txt.strip().splitlines()[-1]
        out[name] = {"N": int(m.group(1)), "n": int(m.group(2)), "m": int(m.group(3)),
                     "values": [float(v) for v in vals_line.replace(",", " ").split()]}
    return {"source": "src/eps/tutorials/output/ex2_1.out (+ _alt)", "args": {"n": 72, "nev": 4, "ncv": 20,
            "which": "largest_magnitude"}, "digits": 5, "outputs": out}


def eps_test2(root):
    """EPS test2: 1-D Laplacian n=30, nev=4, tol=max(1000 eps, 1e-9) = 1e-9, largest and smallest real;
    the same expected output for -eps_type krylovschur -eps_krylovschur_locking {0 1} (test2.c:109-112)."""
    txt = read(root, "src/eps/tests/output/test2_1.out")

    def values(section):
        block = txt.split(section)[1].split("\n", 1)[1].split("- - -")[0]
        line = [ln for ln in block.strip().splitlines() if "," in ln][0]
        return [float(v) for v in line.replace(",", " ").split()]

    return {"source": "src/eps/tests/output/test2_1.out", "args": {"n": 30, "nev": 4, "tol": 1e-9,
            "locking": [0, 1]}, "digits": 5,
            "largest_real": values("Largest eigenvalues"), "smallest_real": values("Smallest eigenvalues")}


def bv_test2(root):
    txt = read(root, "src/sys/classes/bv/tests/output/test2_1.out")
    m = re.search(r"Norm of ones\(n,1\) after orthogonalizing against X: ([0-9.eE+-]+)", txt)
    return {"source": "src/sys/classes/bv/tests/output/test2_1.out", "n": 20, "k": 8,
            "fixture": "X[i+j,j] = (3i+j-2)/(2(i+j+1)) for i<=n/2, i+j<n (test2.c:55-62)",
            "orthogonality_below_100eps": "Level of orthogonality < 100*eps" in txt,
            "norm_ones_after_orth": float(m.group(1)), "digits": 6}


def ds_test2(root):
    txt = read(root, "src/sys/classes/ds/tests/output/test2_1.out")
    block = txt.split("Computed eigenvalues =")[1].split("Value of rnorm")[0]
    eigs = [float(v) for v in block.split()]
    rn = float(re.search(r"rnorm for 3rd vector = ([0-9.]+)", txt).group(1))
    n1 = float(re.search(r"Norm of 1st vector = ([0-9.]+)", txt).group(1))
    return {"source": "src/sys/classes/ds/tests/output/test2_1.out", "n": 12, "ld": 14,
            "fixture": "symmetric Toeplitz: 2 on the diagonal, 1 on the first two off-diagonals (test2.c:47-51)",
            "sort": "largest_magnitude", "eigenvalues": eigs, "rnorm_3rd": rn, "norm_1st": n1}


def _vec_blocks(section):
    blocks = []
    for part in section.split("Vec Object:")[1:]:
        nums = []
        for line in part.splitlines()[2:]:
            line = line.strip()
            if not line:
                continue
            try:
                nums.append(float(line))
            except ValueError:
                break
        blocks.append(nums)
    return blocks


def _mat_rows(section):
    rows = []
    for line in section.splitlines():
        parts = line.split()
        try:
            rows.append([float(p) for p in parts])
        except ValueError:
            continue
    return [r for r in rows if r]


def bv_test1(root):
    txt = read(root, "src/sys/classes/bv/tests/output/test1_1_bv_type-svec.out")
    after_mult = txt.split("After BVMult - - -")[1].split("After BVMultVec")[0]
    after_multvec = txt.split("After BVMultVec - - -")[1].split("After BVDot ")[0]
    after_dot = txt.split("After BVDot - - -")[1].split("After BVDotVec")[0]
    after_dotvec = txt.split("After BVDotVec - - -")[1].split("After BVMultInPlace")[0]
    after_mip = txt.split("After BVMultInPlace - - -")[1].split("2-Norm")[0]
    n2 = float(re.search(r"2-Norm of X\[0\] = ([0-9.]+)", txt).group(1))
    fro = float(re.search(r"Frobenius Norm of X = ([0-9.]+)", txt).group(1))
    return {"source": "src/sys/classes/bv/tests/output/test1_1_bv_type-svec.out", "n": 10, "k": 5, "l": 3,
            "fixture": "X[i+j,j] = 3i+j-2 (i<4); Y[:,j] = (j+1)/4; Q[i,j] = 2 if i<j else -0.5 (test1.c:58-96)",
            "Y_after_mult": _vec_blocks(after_mult), "Y_after_multvec": _vec_blocks(after_multvec),
            "M_after_dot": _mat_rows(after_dot.split("type: seqdense")[1]),
            "z_after_dotvec": _vec_blocks(after_dotvec)[0],
            "X_after_multinplace_scale2": _vec_blocks(after_mip), "norm2_X0": n2, "norm_fro": fro}


def bv_test11(root):
    """test11.c: BVOrthogonalize of columns [0,l) and then [l,k) with each block type; the expected
    output lists the checks that come out below 100 eps (without and with the R factor)."""
    out = {}
    for name, resid in (("test11_1.out", False), ("test11_6.out", True)):
        txt = read(root, "src/sys/classes/bv/tests/output/" + name)
        m = re.search(r"length (\d+), l=(\d+), k=(\d+)", txt)
        out[name] = {"n": int(m.group(1)), "l": int(m.group(2)), "k": int(m.group(3)), "resid": resid,
                     "below_100eps": re.findall(r"^\s+(.*?) < 100\*eps$", txt, flags=re.M)}
    return {"source": "src/sys/classes/bv/tests/output/test11_1.out, test11_6.out",
            "block_types": {"test11_1.out": ["gs", "chol", "tsqr", "tsqrchol", "svqb"],
                            "test11_6.out": ["gs", "chol", "tsqr", "tsqrchol", "svqb"]},
            "fixture": "X[i+j,j] = (3i+j-2)/(2(i+j+1)) for i<=n/2, i+j<n (test11.c:75-91)",
            "outputs": out}


def petsc_binary(root):
    """The two PETSc binary files of ex31 (a Vec and an AIJ Mat), decoded with the published
    layout (big-endian int32 header and indices, float64 values; values kept exactly as hex)."""
    import struct

    out = {}
    raw = open(os.path.join(root, "src/eps/tutorials/X.bin"), "rb").read()
    cid, n = struct.unpack(">ii", raw[:8])
    vals = struct.unpack(">%dd" % n, raw[8:8 + 8 * n])
    out["X.bin"] = {"classid": cid, "n": n, "values_hex": [v.hex() for v in vals], "bytes": len(raw)}
    raw = open(os.path.join(root, "src/eps/tutorials/Ybus.bin"), "rb").read()
    cid, m, ncol, nz = struct.unpack(">iiii", raw[:16])
    off = 16
    lens = struct.unpack(">%di" % m, raw[off:off + 4 * m])
    off += 4 * m
    cols = struct.unpack(">%di" % nz, raw[off:off + 4 * nz])
    off += 4 * nz
    vals = struct.unpack(">%dd" % nz, raw[off:off + 8 * nz])
    out["Ybus.bin"] = {"classid": cid, "m": m, "n": ncol, "nz": nz, "row_lengths": list(lens),
                       "colind": list(cols), "values_hex": [v.hex() for v in vals], "bytes": len(raw)}
    return {"source": "src/eps/tutorials/X.bin, Ybus.bin (read by ex31.c:551-562 with VecLoad / MatLoad)",
            "files": out}


def main(root):
    fixtures = {"ex2_1.json": ex2(root), "eps_test2.json": eps_test2(root), "bv_test2.json": bv_test2(root), "ds_test2.json": ds_test2(root),
                "bv_test1.json": bv_test1(root), "petsc_binary.json": petsc_binary(root),
                "bv_test11.json": bv_test11(root)}
    for name, obj in fixtures.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/slepc")
    main(sys.argv[1])
