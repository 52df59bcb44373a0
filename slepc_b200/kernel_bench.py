"""Single-kernel timing at the 3-D 128^3 Laplacian size (n = 2,097,152) through the C ABI.

Used to produce the kernel profiles (run it under ncu with -k/-s/-c) and to
time one kernel family in isolation with CUDA events:

  python slepc_b200/kernel_bench.py gs --j 20 60    # one column orthogonalisation against j columns
  python slepc_b200/kernel_bench.py spmv             # CSR SpMV of the 7-point Laplacian
  python slepc_b200/kernel_bench.py multinplace      # restart GEMM V(:,0:56) = V(:,0:80) Q
  python slepc_b200/kernel_bench.py cross            # A x, A^T z, A^T A x of the 2M x 500k power-law matrix
  python slepc_b200/kernel_bench.py batched          # the batched Krylov-Schur launch on a small k-NN batch
  python slepc_b200/kernel_bench.py lobpcg --lgrid 512   # LOBPCG per block orthogonalization type
  python slepc_b200/kernel_bench.py mixed            # the mixed-precision solve with per-filter timing
  python slepc_b200/kernel_bench.py rbgram           # the tensor-core and FP64 block Gram products

Prints one JSON line per kernel family: average ms per call and algorithmic GB/s.
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import slepc_b200 as S  # noqa: E402
from slepc_b200 import problems as P  # noqa: E402


def gs(args, torch):
    n, j = args.n, args.j
    bv = S.BV().create(n, args.m)
    rng = np.random.default_rng(0)
    # an orthonormal basis of j columns built by the library itself, then a vector with large components on it
    for c in range(j):
        bv.setColumn(c, rng.standard_normal(n))
        bv.orthonormalizeColumn(c)
    # components along the basis much larger than the rest, as for A*v_j in Lanczos: the first CGS pass
    # leaves |w'| < eta*|w| and the DGKS refinement runs (three streamed passes)
    coeff = 1.0e3 * rng.standard_normal(j)
    base = torch.from_numpy(rng.standard_normal(n)).cuda()
    _, _, ld = bv.getSizes()
    w = base.clone()
    for c in range(0, j, 16):  # w = base + V(:,0:j) coeff, built with BVMultVec on device
        bv.setActiveColumns(c, min(j, c + 16))
        bv.multVec(1.0, 1.0, w.data_ptr(), coeff[c:min(j, c + 16)])
    bv.setActiveColumns(0, args.m)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lib = S.lib()
    for _ in range(args.warmup):
        lib.b200_bv_insert_vec(bv.handle, j, w.data_ptr())
        bv.orthonormalizeColumn(j)
    ms = 0.0
    for _ in range(args.reps):
        lib.b200_bv_insert_vec(bv.handle, j, w.data_ptr())
        torch.cuda.synchronize()
        e0.record()
        nrm, _ = bv.orthonormalizeColumn(j)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= args.reps
    # three streamed passes (dot; update+dot; update+scale) of j basis columns plus w, and two writes of w
    algo = 8 * n * (3 * (j + 1) + 2)
    return {"kernel": "gs_pass_kernel x3 (one column, DGKS refined)", "n": n, "j": j, "ms": ms,
            "algorithmic_bytes": algo, "GBps": algo / (ms * 1e-3) / 1e9, "norm": nrm, "ld": ld}


def spmv(args, torch):
    csr = P.laplacian_3d(args.grid)
    n = len(csr[0]) - 1
    nnz = int(csr[0][-1])
    A = S.Mat().createAIJ(csr)
    A.setSpMVSchedule(args.schedule)
    x = torch.from_numpy(P.start_vector(n, 0)).cuda()
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        A.mult(x.data_ptr(), y.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(args.reps):
        flush.fill_(1.0)  # evict x and the CSR arrays from L2 between calls
        e0.record()
        A.mult(x.data_ptr(), y.data_ptr())
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= args.reps
    algo = nnz * 12 + (n + 1) * 4 + 2 * n * 8
    return {"kernel": ["spmv_rowblock_kernel", "spmv_warptile_kernel", "spmv_warptile_pipelined_kernel", "spmv_sell_kernel"][args.schedule], "n": n, "nnz": nnz, "ms": ms, "algorithmic_bytes": algo,
            "GBps": algo / (ms * 1e-3) / 1e9}


def spmm(args, torch):
    """BVMatMult of the 3-D Laplacian on a block of --nb columns (the block SpMV of the mixed
    solver's refinement phase), L2 flushed between calls."""
    csr = P.laplacian_3d(args.grid)
    n = len(csr[0]) - 1
    nnz = int(csr[0][-1])
    A = S.Mat().createAIJ(csr)
    nb = args.nb
    V = S.BV().create(n, nb)
    Y = S.BV().create(n, nb)
    rng = np.random.default_rng(0)
    for j in range(nb):
        V.setColumn(j, rng.standard_normal(n))
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        V.matMult(A, Y)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(args.reps):
        flush.fill_(1.0)
        e0.record()
        V.matMult(A, Y)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= args.reps
    algo = nnz * 12 + (n + 1) * 4 + 2 * nb * n * 8
    return {"kernel": "spmm_sell_kernel (BVMatMult)", "n": n, "nnz": nnz, "columns": nb, "ms": ms,
            "algorithmic_bytes": algo, "GBps": algo / (ms * 1e-3) / 1e9}


def mixed(args, torch):
    """The mixed-precision solve of the 3-D Laplacian (nev 32, ncv 80, tol 1e-8) with per-filter timing:
    the solver's counters and the block SpMV's algorithmic GB/s (device-counted bytes over the CUDA-event
    time of the filters)."""
    csr = P.laplacian_3d(args.grid)
    n = len(csr[0]) - 1
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setDimensions(32, 80)
    E.setTolerances(1e-8)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    E.setInitialSpace(P.start_vector(n, 0))
    E.setPrecision(S.EPS.Precision.MIXED)
    if args.fp64_gram:
        E.setMixedOptions(fp64_gram=True)
    E.solve()
    E.setTiming(True)
    E.solve()
    st = E.getStats()
    nconv = E.getConverged()
    err = max(E.computeError(i) for i in range(min(nconv, 32))) if nconv else None
    E.destroy()
    A.destroy()
    gbs = st["gs_bytes"] / (st["ms_spmv"] * 1e-3) / 1e9 if st["ms_spmv"] > 0 else None
    return {"kernel": "mixed solve (Chebyshev-filtered block, FP32 then FP64)", "n": n, "nconv": nconv,
            "max_rel_residual": err, "filter_GBps": gbs, **st}


def rbgram(args, torch):
    """G = X^T X and X^T Y of n x 64 row-major FP32 blocks through b200_rowblock_gram (tensor cores and
    FP64), each call timed with CUDA events (the call also allocates and frees its work arrays)."""
    n, bp = args.n, 64
    X = torch.randn((n, bp), dtype=torch.float32, device="cuda")
    Y = torch.randn((n, bp), dtype=torch.float32, device="cuda")
    G = torch.empty((bp, bp), dtype=torch.float64, device="cuda")
    out = []
    for tc in (True, False):
        for cross in (False, True):
            yp = Y.data_ptr() if cross else None
            for _ in range(args.warmup):
                S.rowblock_gram(n, bp, X.data_ptr(), yp, tc, G.data_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ms = 0.0
            for _ in range(args.reps):
                torch.cuda.synchronize()
                e0.record()
                S.rowblock_gram(n, bp, X.data_ptr(), yp, tc, G.data_ptr())
                e1.record()
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
            ms /= args.reps
            algo = n * bp * 4 * (2 if cross else 1)
            out.append({"kernel": ("rb_gram_tf32_kernel (tcgen05)" if tc else "rb_gram2_kernel (FP64)") +
                        (" X^T Y" if cross else " X^T X"), "n": n, "bp": bp, "ms_per_call": ms,
                        "algorithmic_bytes": algo, "GBps_call": algo / (ms * 1e-3) / 1e9})
    return out


def lobpcg(args, torch):
    """LOBPCG (smallest 16, block 16, Jacobi) on the 2-D anisotropic diffusion operator of an
    --lgrid^2 grid, once per BVOrthogBlockType: iterations, seconds, milliseconds and kernel
    launches per iteration, and the largest eigenvalue difference from the Gram-Schmidt run."""
    from slepc_b200 import learned

    csr = P.diffusion_problem(args.lgrid, 1)[0]
    out, base = [], None
    for name in args.block:
        t = {"gs": S.BV.OrthogBlockType.GS, "chol": S.BV.OrthogBlockType.CHOL, "svqb": S.BV.OrthogBlockType.SVQB}[name]
        learned.solve_lowest(S, csr, nev=16, max_it=3, orthog_block=t)  # warm-up: allocations, first launches
        r = learned.solve_lowest(S, csr, nev=16, orthog_block=t, stats=True)
        if base is None:
            base = r["vals"]
        its = max(r["its"], 1)
        line = {"kernel": f"lobpcg orthog_block={name}", "n": args.lgrid ** 2, "its": r["its"],
                "reason": r["reason"], "seconds": round(r["seconds"], 4),
                "ms_per_iteration": round(1e3 * r["seconds"] / its, 4),
                "launches_per_iteration": round(r["stats"]["kernel_launches"] / its, 1),
                "max_error": r["max_error"],
                "max_rel_diff_vs_first": float(np.max(np.abs(r["vals"] - base) / np.abs(base)))}
        if args.phases:
            # a second run with the phase edges synchronised: where an iteration's time goes
            q = learned.solve_lowest(S, csr, nev=16, orthog_block=t, stats=True, timing=True)
            st, qi = q["stats"], max(q["its"], 1)
            line["phase_ms_per_iteration"] = {k: round(st[f"ms_{k}"] / qi, 4) for k in ("spmv", "orth", "restart",
                                                                                          "total")}
        out.append(line)
    return out


def lobpcg_ops(args, torch):
    """The block operations of one LOBPCG iteration at n = --lgrid^2, each timed alone on the host
    clock over --reps x 20 calls (every call ends with a read-back or a synchronisation, as in the
    solver): BVDot of 48-column blocks, BVMult 32 -> 16 columns, BVOrthogonalize of 16 columns per
    block type, the host generalized eigensolve of a 48 x 48 pencil, and an empty synchronisation."""
    import time

    import scipy.linalg as sl

    n = args.lgrid ** 2
    rng = np.random.default_rng(0)
    Z = S.BV().create(n, 48)
    W = S.BV().create(n, 48)
    Z.setColumns(rng.standard_normal((n, 48)))
    W.setColumns(rng.standard_normal((n, 48)))
    P16 = S.BV().create(n, 16)
    Q = rng.standard_normal((48, 16))
    out = []

    def timed(name, fn, calls=20):
        fn()
        best = None
        for _ in range(args.reps):
            t0 = time.perf_counter()
            for _ in range(calls):
                fn()
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) / calls * 1e3
            best = dt if best is None else min(best, dt)
        out.append({"op": name, "n": n, "ms_per_call": round(best, 4)})

    timed("BVDot 48 x 48", lambda: W.dot(Z))
    Z.setActiveColumns(16, 48)
    timed("BVMult 32 -> 16 (beta 0)", lambda: P16.mult(1.0, 0.0, Z, Q))
    timed("BVMult 32 -> 16 (beta 1)", lambda: P16.mult(1.0, 1.0, Z, Q))
    Z.setActiveColumns(0, 48)
    for name, t in (("gs", S.BV.OrthogBlockType.GS), ("chol", S.BV.OrthogBlockType.CHOL),
                    ("svqb", S.BV.OrthogBlockType.SVQB)):
        R = S.BV().create(n, 16)
        R.setColumns(rng.standard_normal((n, 16)))
        R.setOrthogonalizationBlock(t)
        timed(f"BVOrthogonalize 16 columns ({name})", lambda: R.orthogonalize(16))
        R.destroy()
    A = rng.standard_normal((48, 48))
    A = A + A.T
    B = rng.standard_normal((48, 48))
    B = B @ B.T + 48 * np.eye(48)
    timed("host dsygvd 48 x 48 (scipy)", lambda: sl.eigh(A, B, driver="gvd"))
    timed("empty stream synchronisation", lambda: torch.cuda.synchronize())
    return out


def cross(args, torch):
    """A x and A^T z of the power-law rectangular matrix (FP32 values), each timed alone with L2
    flushed, plus the A^T A shell."""
    m, n = args.rows, args.cols
    rowptr, colind, vals = P.powerlaw_rect(m, n, 20, 1.8, seed=0)
    nnz = int(rowptr[-1])
    A = S.Mat().createAIJ((rowptr, colind, vals), size=(m, n), dtype=np.float32)
    C = S.Mat().createCross(A)
    x = torch.from_numpy(P.start_vector(n, 0)).cuda()
    z = torch.from_numpy(P.start_vector(m, 1)).cuda()
    y = torch.empty(m, dtype=torch.float64, device="cuda")
    yt = torch.empty(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms = 0.0
        for _ in range(args.reps):
            flush.fill_(1.0)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / args.reps

    ms_a = timed(lambda: A.mult(x.data_ptr(), y.data_ptr()))
    ms_at = timed(lambda: A.multTranspose(z.data_ptr(), yt.data_ptr()))
    ms_c = timed(lambda: C.mult(x.data_ptr(), yt.data_ptr()))
    part = lambda rows, cols: nnz * 8 + (rows + 1) * 4 + cols * 8 + rows * 8
    out = []
    for name, ms, algo in [("A x (warp tiles, 20 nonzeros per row)", ms_a, part(m, n)),
                           ("A^T z (segments of the power-law columns)", ms_at, part(n, m)),
                           ("A^T (A x) shell", ms_c, part(m, n) + part(n, m))]:
        out.append({"kernel": name, "m": m, "n": n, "nnz": nnz, "ms": ms, "algorithmic_bytes": algo,
                    "GBps": algo / (ms * 1e-3) / 1e9})
    return out


def batched(args, torch):
    """The batched Krylov-Schur launch on a small k-NN batch (n ~ U[500, 3000]); device time per solve
    and the device-counted algorithmic bytes."""
    ns = P.batch_sizes(args.nprob, 1, 500, 3000)
    B = P.knn_batch(ns, 8, 1)
    v0 = np.concatenate([P.start_vector(int(n), p) for p, n in enumerate(ns)])
    E = S.BatchEPS().create(B.ns, B.rowptr, B.colind, B.vals)
    E.setDimensions(8, 24)
    E.setInitialVectors(v0)
    E.setThreads(args.threads)
    for _ in range(args.warmup):
        E.solve()
    ms = 0.0
    for _ in range(args.reps):
        E.solve()
        ms += E.getAll()[2]
    ms /= args.reps
    algo = E.getBytes()
    return {"kernel": "batched_ks_kernel", "nprob": args.nprob, "rows": int(ns.sum()), "threads": args.threads,
            "ms": ms, "algorithmic_bytes": algo, "GBps": algo / (ms * 1e-3) / 1e9}


def multinplace(args, torch):
    n, k, e = args.n, 80, 56
    bv = S.BV().create(n, 81)
    rng = np.random.default_rng(1)
    for c in range(k):
        bv.setColumn(c, rng.standard_normal(n))
    Q = np.asfortranarray(rng.standard_normal((81, 81)))
    bv.setActiveColumns(0, k)
    for _ in range(args.warmup):
        bv.multInPlace(Q, 0, e)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(args.reps):
        torch.cuda.synchronize()
        e0.record()
        bv.multInPlace(Q, 0, e)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= args.reps
    algo = 8 * n * (k + e) + 8 * k * e
    flops = 2.0 * n * k * e
    return {"kernel": "BVMultInPlace (panel_dmma16_kernel, mma.sync m16n8k16 f64)", "n": n, "k": k, "e-s": e, "ms": ms, "algorithmic_bytes": algo,
            "GBps": algo / (ms * 1e-3) / 1e9, "TFLOPs": flops / (ms * 1e-3) / 1e12}


def neural(args, torch):
    """One Adam training step of the neural operator (width 32, 12 x 12 modes, 4 layers, hidden 64,
    16 outputs) on a batch of --nb synthetic fields of --lgrid^2 cells: device time per step and its
    launches (the contractions are tensor-core GEMMs)."""
    N, B = args.lgrid, args.nb
    dims = (N, 32, 12, 4, 64, 16)
    op = S.NeuralOperator().create(*dims)
    from slepc_b200 import learned as LN

    op.setParams(LN.init_params(*dims, seed=0))
    g = torch.Generator(device="cuda").manual_seed(0)
    F = torch.randn((B, 3, N * N), generator=g, device="cuda", dtype=torch.float32)
    T = torch.randn((B, 16, N * N), generator=g, device="cuda", dtype=torch.float32)
    for _ in range(args.warmup):
        op.trainStep(F, T, 1e-4)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = S.kernel_launch_count()
    e0.record()
    for _ in range(args.reps):
        op.trainStep(F, T, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    launches = (S.kernel_launch_count() - l0) / args.reps
    op.destroy()
    return {"kernel": "neural-operator training step (forward, loss, backward, Adam)", "grid": N, "batch": B,
            "ms": ms, "launches_per_step": launches, "ms_per_field": ms / B}


def tcgemm(args, torch):
    """The neural operator's two heaviest GEMM shapes on a --lgrid^2 grid, batch --nb, width 32, on
    the tensor cores (b200_tc_sgemm_async, CUDA events on the launching stream, L2 flushed between
    calls): the channel mix Out[b] = W In[b]
    (32 x 32 times 32 x P per sample) and the weight gradient dW = sum_b D[b] X[b]^T (32 x 32 from
    two 32 x P blocks per sample); algorithmic bytes = every operand read once and C written once."""
    P_, B, W = args.lgrid ** 2, args.nb, 32
    g = torch.Generator(device="cuda").manual_seed(0)
    In = torch.randn((B, W, P_), generator=g, device="cuda")
    D = torch.randn((B, W, P_), generator=g, device="cuda")
    Wt = torch.randn((W, W), generator=g, device="cuda")
    Out = torch.empty((B, W, P_), device="cuda")
    dW = torch.empty((W, W), device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms = 0.0
        for _ in range(args.reps):
            flush.fill_(1.0)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / args.reps

    ws = torch.empty(1 << 22, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    mix = lambda: S.tc_sgemm_async(B, W, P_, W, 1.0, (Wt.data_ptr(), W, 1, 0), (In.data_ptr(), P_, 1, W * P_), 0.0,
                                   (Out.data_ptr(), P_, 1, W * P_), ws.data_ptr(), ws.numel(), err.data_ptr(),
                                   stream=stream)
    wgrad = lambda: S.tc_sgemm_async(B, W, W, P_, 1.0, (D.data_ptr(), P_, 1, W * P_), (In.data_ptr(), 1, P_, W * P_),
                                     0.0, (dW.data_ptr(), W, 1, 0), ws.data_ptr(), ws.numel(), err.data_ptr(),
                                     sum_batch=True, stream=stream)
    out = []
    for name, fn, algo in [("mix Out[b] = W In[b]", mix, 4 * (2 * B * W * P_ + W * W)),
                           ("weight gradient sum_b D[b] X[b]^T", wgrad, 4 * (2 * B * W * P_ + W * W))]:
        ms = timed(fn)
        out.append({"kernel": f"tc_sgemm_kernel: {name}", "grid": args.lgrid, "batch": B, "ms": ms,
                    "algorithmic_bytes": algo, "GBps": algo / (ms * 1e-3) / 1e9})
    torch.cuda.synchronize()
    if int(err.item()) != 0:
        raise RuntimeError(f"tensor-core GEMM error bits {int(err.item())}")
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("kernel", choices=["gs", "spmv", "spmm", "mixed", "rbgram", "multinplace", "cross", "batched", "lobpcg",
                                      "lobpcg_ops", "neural", "tcgemm", "all"])
    p.add_argument("--lgrid", type=int, default=512, help="lobpcg: side of the 2-D diffusion grid")
    p.add_argument("--block", nargs="+", default=["gs", "chol", "svqb"], help="lobpcg: block orthogonalizations")
    p.add_argument("--phases", action="store_true", help="lobpcg: also a run with per-phase times")
    p.add_argument("--fp64-gram", action="store_true", help="mixed: FP64 orthonormalisation Gram (no tensor cores)")
    p.add_argument("--nb", type=int, default=48, help="columns of the BVMatMult block")
    p.add_argument("--nprob", type=int, default=64)
    p.add_argument("--threads", type=int, default=512)
    p.add_argument("--rows", type=int, default=2_000_000)
    p.add_argument("--cols", type=int, default=500_000)
    p.add_argument("--n", type=int, default=128 ** 3)
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--j", type=int, nargs="+", default=[60])
    p.add_argument("--m", type=int, default=82)
    p.add_argument("--reps", type=int, default=5)
    p.add_argument("--schedule", type=int, default=1, help="SpMV schedule: 0 row blocks, 1 warp tiles")
    p.add_argument("--warmup", type=int, default=2)
    args = p.parse_args()
    import torch

    todo = ["gs", "spmv", "multinplace"] if args.kernel == "all" else [args.kernel]
    js = list(args.j)
    for k in todo:
        if k == "gs":
            for j in js:
                args.j = j
                print(json.dumps(gs(args, torch)), flush=True)
        elif k == "batched":
            print(json.dumps(batched(args, torch)), flush=True)
        elif k in ("lobpcg", "lobpcg_ops"):
            for line in (lobpcg if k == "lobpcg" else lobpcg_ops)(args, torch):
                print(json.dumps(line), flush=True)
        elif k in ("cross", "rbgram", "tcgemm"):
            for line in {"cross": cross, "rbgram": rbgram, "tcgemm": tcgemm}[k](args, torch):
                print(json.dumps(line), flush=True)
        else:
            print(json.dumps({"spmv": spmv, "spmm": spmm, "mixed": mixed, "multinplace": multinplace,
                              "neural": neural}[k](args, torch)),
                  flush=True)


if __name__ == "__main__":
    main()
