#!/usr/bin/env python
"""Benchmark of the B200 Krylov-Schur eigensolver on the 3-D 128^3 Laplacian
(default), or of the SVD cross solver on a power-law rectangular matrix
(--workload cross).

Workload (one "step" = one full EPSSolve from the seeded start vector):
  3-D 7-point Dirichlet Laplacian on a 128^3 grid (n = 2,097,152, 14,581,760
  nonzeros, FP64 CSR), nev = 32 largest real, ncv = 80, tol = 1e-8, start
  vector N(0,1) from seed 0.  Metric: seconds until every requested residual
  is <= 1e-8 (lower is better), plus the HBM bandwidth of the dominant kernel.

  --impl b200       the CUDA library (default)
  --impl reference  the CPU oracle (a restatement of SLEPc's EPSSolve, which
                    itself cannot be built here without PETSc) on all host
                    cores, on a bounded sample of the workload extrapolated
                    to the full solve.

Multi-GPU (torchrun): every rank solves its own replica of the single-problem
workloads; the batched workload is sharded by problem (each rank solves its
contiguous share of the batch, no data-path collective).  Timings are the max
over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from slepc_b200 import problems as P  # noqa: E402

# The oracle's complete solve of the default workload (tests/golden/make_laplacian3d_fixture.py,
# 8 threads): Gram-Schmidt column visits (sum over Lanczos steps j of j+2), iterations and Lanczos
# steps.  The reference arm extrapolates its bounded CPU sample by these column visits, the quantity
# its dominant work is linear in; the complete solve measured 363 s on 8 threads of a 2.7 GHz Xeon.
FULL_SOLVE_COLUMN_VISITS = {128: 216778}
FULL_SOLVE_ORACLE = {128: {"its": 101, "lanczos_steps": 3385, "column_visits": 216778, "wall_s_8_threads": 363.0}}
# Lanczos steps of a full solve of the SVD cross workload (rows, cols, nsv, ncv), measured by the GPU arm.
FULL_SOLVE_LANCZOS_STEPS_CROSS = {}

SPMV_BYTES_PER_NNZ = 12  # 8-byte value + 4-byte column index


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--nev", type=int, default=32)
    p.add_argument("--ncv", type=int, default=80)
    p.add_argument("--cpu-restarts", type=int, default=4, help="restarts in the bounded CPU sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                   help="laplacian3d: arithmetic of the timed solve (fp64: the drop-in path; mixed: FP32 basis "
                        "then FP64 Chebyshev-filtered Rayleigh-Ritz); the fp64 line also reports the mixed form")
    p.add_argument("--learn-grid", type=int, default=64, help="learned workload: N of the N x N diffusion grid")
    p.add_argument("--learn-nev", type=int, default=16, help="learned workload: eigenpairs (LOBPCG block)")
    p.add_argument("--train-fields", type=int, default=256, help="learned workload: training fields")
    p.add_argument("--eval-fields", type=int, default=16,
                   help="learned workload: held-out fields per step (every step, warm-up included, its own)")
    p.add_argument("--epochs", type=int, default=120, help="learned workload: training epochs")
    p.add_argument("--learn-orthog", choices=["gs", "chol"], default="chol",
                   help="learned workload: block orthogonalization of the LOBPCG solves (BVOrthogBlockType)")
    p.add_argument("--learn-modes", type=int, default=12, help="learned workload: sine modes per direction")
    p.add_argument("--e2e-steps", type=int, default=0,
                   help="learned workload: timed steps repeated end to end (0: all of them)")
    p.add_argument("--cpu-max-it", type=int, default=0,
                   help="learned workload: iterations of the oracle's CPU sample (0: a complete solve); the "
                        "per-iteration time is scaled by the GPU solve's iterations from the random block")
    p.add_argument("--workload", choices=["laplacian3d", "cross", "batched", "learned"], default="laplacian3d",
                   help="laplacian3d: the EPS headline case; cross: largest singular triplets of the "
                        "2,000,000 x 500,000 power-law matrix through A^T A; batched: 4096 k-NN graph "
                        "eigenproblems in one persistent launch")
    p.add_argument("--nprob", type=int, default=4096, help="batched workload: number of problems")
    p.add_argument("--cpu-sample", type=int, default=256, help="batched workload: problems in the CPU sample")
    p.add_argument("--rows", type=int, default=2_000_000, help="cross workload: rows of A")
    p.add_argument("--cols", type=int, default=500_000, help="cross workload: columns of A")
    p.add_argument("--nsv", type=int, default=32, help="cross workload: singular triplets")
    p.add_argument("--svd-ncv", type=int, default=96, help="cross workload: ncv")
    p.add_argument("--svd-dtype", choices=["f32", "f64"], default="f32", help="cross workload: value storage")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM traffic of the Gram-Schmidt pass kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "gs_pass_kernel_128cubed.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_algorithmic_byte:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


def workload(grid):
    csr = P.laplacian_3d(grid)
    n = len(csr[0]) - 1
    return csr, n, P.start_vector(n, 0)


def config_dict(args, n, nnz, extra=None):
    form = ("FP64 CSR, Krylov-Schur (CGS+DGKS, thick restart)" if args.precision == "fp64" else
            "FP64 CSR, mixed form: Chebyshev-filtered subspace iteration on a 64-vector row-major block, FP32 block "
            "and FP32 matrix values (orthonormalisation Gram on the tensor cores, TF32 with FP32 accumulation; "
            "Rayleigh quotients and residuals in FP64) to 5e-7, then the same sweeps in FP64 to 1e-8")
    d = {"workload": f"3-D 7-point Laplacian {args.grid}^3, nev={args.nev} largest real, ncv={args.ncv}, tol=1e-8, "
                     + form,
         "n": n, "nnz": nnz, "nev": args.nev, "ncv": args.ncv, "tol": 1e-8, "start_vector": "N(0,1) seed 0",
         "l2": "inputs larger than L2: basis V is n x 81 FP64 = %.2f GB, CSR %.0f MB (L2 = 126 MB)"
               % (n * 81 * 8 / 1e9, (nnz * 12 + (n + 1) * 4) / 1e6),
         "parallelism": "replicas" if args.gpus > 1 else "single GPU"}
    if extra:
        d.update(extra)
    return d


def cpu_sample(csr, v0, args, threads):
    import oracle

    oracle.set_threads(threads)
    A = P.to_scipy(csr)
    t0 = time.perf_counter()
    r = oracle.eps_solve(A, v0, nev=args.nev, ncv=args.ncv, which=oracle.LARGEST_REAL,
                         max_restarts=args.cpu_restarts, want_vectors=False)
    t = time.perf_counter() - t0
    return t, r


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    csr, n, v0 = workload(args.grid)
    threads = os.cpu_count() or 1
    full_visits = FULL_SOLVE_COLUMN_VISITS.get(args.grid)
    if full_visits is None:
        print(json.dumps({"impl": "reference", "unavailable": "no full-solve column count recorded for this grid"}))
        return 0
    for _ in range(args.warmup):
        cpu_sample(csr, v0, args, threads)
    times, visits = [], None
    for _ in range(args.steps):
        t, r = cpu_sample(csr, v0, args, threads)
        times.append(t)
        visits = r.column_visits
    per_visit = statistics.mean(times) / visits
    value = per_visit * full_visits
    sample = (f"first {args.cpu_restarts} restart(s) of the solve ({visits} Gram-Schmidt column visits, "
              f"{statistics.mean(times):.1f} s), extrapolated to the {full_visits} column visits of a full solve")
    line = {"impl": "reference", "metric": "time_to_all_residuals_le_1e-8", "value": value, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated 3-D Laplacian, seeded N(0,1) start vector)",
            "config": config_dict(args, n, int(csr[0][-1])),
            "solve": dict(FULL_SOLVE_ORACLE.get(args.grid, {}), source="the oracle's complete solve of this workload"),
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_b200(args):
    import torch

    import slepc_b200 as S

    from slepc_b200.ranks import Ranks

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    ranks = Ranks("nccl", timeout_s=600)  # replicas: barrier and max over ranks, no data-path collective
    barrier, max_over_ranks = ranks.barrier, ranks.max

    csr, n, v0 = workload(args.grid)
    nnz = int(csr[0][-1])
    A = S.Mat().createAIJ(csr)
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setDimensions(args.nev, args.ncv)
    E.setTolerances(1e-8)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    mixed = args.precision == "mixed"
    if mixed:
        E.setPrecision(S.EPS.Precision.MIXED)
    # start vector resident in HBM: the timed region starts with inputs on the device
    v0_dev = torch.from_numpy(v0).cuda()
    E.setInitialSpaceDevice(v0_dev.data_ptr())

    for _ in range(args.warmup):
        E.solve()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = S.kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        E.solve()
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = S.kernel_launch_count() - launches0
    ms_per_step = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)

    # correctness of what was timed: every requested pair converged, residuals in FP64 on the device
    nconv = E.getConverged()
    reason = E.getConvergedReason()
    resid = [E.computeError(i) for i in range(nconv)]
    stats = E.getStats()

    # roofline of the dominant kernel (the fused Gram-Schmidt pass): one more solve with per-phase events
    E.setTiming(True)
    E.solve()
    tstats = E.getStats()
    E.setTiming(False)
    peak, peak_kind = measured_peaks()
    if mixed:
        # the dominant kernel is the filter's block SpMV: device-counted algorithmic bytes / its time
        gs_gbs = tstats["gs_bytes"] / (tstats["ms_spmv"] * 1e-3) / 1e9 if tstats["ms_spmv"] > 0 else None
        spmv_gbs = None
    else:
        gs_gbs = tstats["gs_bytes"] / (tstats["ms_orth"] * 1e-3) / 1e9 if tstats["ms_orth"] > 0 else None
        spmv_bytes = nnz * SPMV_BYTES_PER_NNZ + (n + 1) * 4 + 2 * n * 8
        spmv_gbs = (spmv_bytes * tstats["lanczos_steps"] / (tstats["ms_spmv"] * 1e-3) / 1e9
                    if tstats["ms_spmv"] > 0 else None)
    tr = profiled_traffic()

    # end to end through the one-call host API: host CSR + start vector in, eigenpairs out
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_csr = (pin(csr[0]), pin(csr[1]), pin(csr[2]))
    h_v0 = pin(v0)
    # the caller's page-locked output block, allocated once and reused by every call
    h_out = torch.empty((args.ncv + 1 if not mixed else max(args.ncv + 1, 128), n),
                        dtype=torch.float64).pin_memory().numpy()
    form = S.EPS.Precision.MIXED if mixed else S.EPS.Precision.FP64
    # one untimed call first, as a service would have made: the library's device pool then holds the
    # mixed form's blocks for the timed calls (the FP64 form allocates per call either way)
    S.solve_csr_host(h_csr, h_v0, args.nev, args.ncv, tol=1e-8, which=S.LARGEST_REAL, out=h_out, precision=form)
    barrier()
    t0 = time.perf_counter()
    e2e_last = None
    for _ in range(args.steps):
        e2e_last = S.solve_csr_host(h_csr, h_v0, args.nev, args.ncv, tol=1e-8, which=S.LARGEST_REAL, out=h_out,
                                    precision=form)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    h2d = csr[0].nbytes + csr[1].nbytes + csr[2].nbytes + v0.nbytes
    d2h = e2e_last["nconv"] * (n * 8 + 16)

    # the other form, device-timed outside the timed region: the mixed form beside the FP64 line
    mixed_line = None
    if not mixed:
        plain_vals = np.array([E.getEigenpair(i, want_vector=False) for i in range(min(nconv, args.nev))])
        mixed_line = measure_mixed(S, torch, A, v0_dev, args, plain_vals, ms_per_step)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t, r = cpu_sample(csr, v0, args, threads)
        visits = stats["column_visits"] or FULL_SOLVE_COLUMN_VISITS.get(args.grid, r.column_visits)
        value = t / r.column_visits * visits
        cpu = {"value": value, "unit": "s", "cores": threads, "kind": "port",
               "sample": (f"first {args.cpu_restarts} restart(s) of the same solve on {threads} host threads "
                          f"({r.column_visits} Gram-Schmidt column visits in {t:.1f} s), extrapolated to the "
                          f"{visits} column visits of the full FP64 solve")}

    if rank == 0:
        line = {"metric": "time_to_all_residuals_le_1e-8", "value": ms_per_step / 1e3, "unit": "s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 block then f64" if mixed else "f64",
                "data": "synthetic (generated 3-D Laplacian, seeded N(0,1) start vector)",
                "config": config_dict(args, n, nnz),
                "solve": ({"fp32_sweeps": stats["phase1_restarts"], "fp64_sweeps": stats["filter_sweeps"],
                           "block_size": stats["block_size"], "block_spmv_columns": stats["spmm_columns"],
                           "max_degree": stats["filter_degree"], "ms_fp32_phase": stats["ms_phase1"],
                           "ms_fp64_phase": stats["ms_phase2"]} if mixed else
                          {"restarts": stats["restarts"], "lanczos_steps": stats["lanczos_steps"],
                           "gs_passes": stats["gs_passes"], "column_visits": stats["column_visits"]}) | {
                    "nconv": nconv, "reason": reason, "max_rel_residual": max(resid) if resid else None},
                "roofline": {"kernel": ("rb_spmm_kernel (row-major block SpMV with the fused Chebyshev three-term "
                                        "update, FP32 and FP64 phases)"
                                        if mixed else "gs_pass_kernel (fused CGS update+dot, DGKS on device)"),
                             "bound": "hbm",
                             "achieved": gs_gbs, "peak": peak, "unit": "GB/s",
                             "frac": (gs_gbs / peak) if gs_gbs else None,
                             "peak_kind": peak_kind,
                             "traffic": (tr * tstats["gs_bytes"] / max(tstats["gs_passes"], 1)) if tr and not mixed
                             else None,
                             "spmv_achieved": spmv_gbs, "spmv_frac": (spmv_gbs / peak) if spmv_gbs else None,
                             "share_orth": (tstats["ms_orth"] / tstats["ms_total"] if tstats["ms_total"] and not mixed
                                            else None),
                             "share_spmv": tstats["ms_spmv"] / tstats["ms_total"] if tstats["ms_total"] else None,
                             "share_restart": tstats["ms_restart"] / tstats["ms_total"] if tstats["ms_total"] else None},
                "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(launches),
                "clocks": clk,
                "cpu_baseline": cpu}
        if mixed_line is not None:
            line["mixed"] = mixed_line
        print(json.dumps(line))
    E.destroy()
    A.destroy()
    ranks.close()
    return 0


def measure_mixed(S, torch, A, v0_dev, args, plain_vals, plain_ms):
    """The mixed form on the same matrix and start vector: device time per solve (CUDA events, one
    warm-up), residuals in FP64, and the error of each eigenvalue against the FP64 run and against
    the exact spectrum of the Laplacian."""
    E = S.EPS().create()
    E.setOperators(A)
    E.setProblemType(S.EPS.ProblemType.HEP)
    E.setDimensions(args.nev, args.ncv)
    E.setTolerances(1e-8)
    E.setWhichEigenpairs(S.LARGEST_REAL)
    E.setPrecision(S.EPS.Precision.MIXED)
    E.setInitialSpaceDevice(v0_dev.data_ptr())
    E.solve()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        E.solve()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    st = E.getStats()
    nconv = min(E.getConverged(), args.nev)
    vals = np.array([E.getEigenpair(i, want_vector=False) for i in range(nconv)])
    resid = [E.computeError(i) for i in range(nconv)]
    E.setTiming(True)
    E.solve()
    ts = E.getStats()
    E.destroy()
    exact = np.sort(P.laplacian_3d_eigs(args.grid))[::-1][: args.nev]
    m = min(len(vals), len(plain_vals))
    rel_fp64 = (np.abs(np.sort(vals)[::-1][:m] - np.sort(plain_vals)[::-1][:m]) /
                np.abs(np.sort(plain_vals)[::-1][:m]))
    return {"value": ms / 1e3, "unit": "s", "ms_per_step": ms, "speedup_vs_fp64": plain_ms / ms,
            "nconv": nconv, "max_rel_residual": max(resid) if resid else None,
            "fp32_sweeps": st["phase1_restarts"], "fp64_sweeps": st["filter_sweeps"],
            "filter_degree": st["filter_degree"], "block_size": st["block_size"],
            "ms_phase1": st["ms_phase1"], "ms_phase2": st["ms_phase2"], "block_spmv_columns": st["spmm_columns"],
            "filter_spmv_achieved_GBps": (ts["gs_bytes"] / (ts["ms_spmv"] * 1e-3) / 1e9) if ts["ms_spmv"] > 0 else None,
            "filter_share_of_solve": (ts["ms_spmv"] / ts["ms_total"]) if ts["ms_total"] > 0 else None,
            "per_pair_rel_err_vs_fp64_run": [float(x) for x in rel_fp64],
            "max_rel_err_vs_fp64_run": float(rel_fp64.max()) if m else None,
            "max_abs_err_vs_exact_top_nev": float(np.abs(np.sort(vals)[::-1] - exact[: len(vals)]).max()),
            "fp64_max_abs_err_vs_exact_top_nev": float(np.abs(np.sort(plain_vals)[::-1] - exact[: len(plain_vals)]).max()),
            "note": ("eigenvalue sets compared sorted; both runs hold every residual below 1e-8, and where the sets "
                     "differ a run found a different number of copies of a repeated eigenvalue")}


# ------------------------------------------------------------------ SVD cross workload
SVD_TOL = 1e-7


def cross_workload(args):
    csr = P.powerlaw_rect(args.rows, args.cols, 20, 1.8, seed=0)
    return csr, P.start_vector(min(args.rows, args.cols), 0)


def cross_config(args, nnz, extra=None):
    d = {"workload": f"largest {args.nsv} singular triplets of a {args.rows} x {args.cols} sparse matrix "
                     f"(20 distinct columns per row, column index power law exponent 1.8, N(0,1) values stored "
                     f"{'FP32' if args.svd_dtype == 'f32' else 'FP64'}), SVD cross: Krylov-Schur on A^T A, "
                     f"ncv={args.svd_ncv}, tol={SVD_TOL:g}",
         "m": args.rows, "n": args.cols, "nnz": nnz, "nsv": args.nsv, "ncv": args.svd_ncv, "tol": SVD_TOL,
         "start_vector": "N(0,1) seed 0",
         "l2": "inputs larger than L2: A and its transpose %.0f MB, basis %.2f GB (L2 = 126 MB)"
               % (2 * nnz * (8 if args.svd_dtype == "f32" else 12) / 1e6, args.cols * (args.svd_ncv + 1) * 8 / 1e9),
         "parallelism": "replicas" if args.gpus > 1 else "single GPU"}
    if extra:
        d.update(extra)
    return d


def cross_cpu_sample(csr, v0, args, threads):
    import oracle

    oracle.set_threads(threads)
    t0 = time.perf_counter()
    r = oracle.svd_cross(csr[0], csr[1], csr[2].astype(np.float64), (args.rows, args.cols), v0, args.nsv,
                         args.svd_ncv, tol=SVD_TOL, max_restarts=args.cpu_restarts)
    return time.perf_counter() - t0, r


def run_reference_cross(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    csr, v0 = cross_workload(args)
    threads = os.cpu_count() or 1
    full_steps = FULL_SOLVE_LANCZOS_STEPS_CROSS.get((args.rows, args.cols, args.nsv, args.svd_ncv))
    if full_steps is None:
        print(json.dumps({"impl": "reference", "unavailable": "no full-solve Lanczos step count recorded"}))
        return 0
    for _ in range(args.warmup):
        cross_cpu_sample(csr, v0, args, threads)
    times, steps = [], None
    for _ in range(args.steps):
        t, r = cross_cpu_sample(csr, v0, args, threads)
        times.append(t)
        steps = r.lanczos_steps
    value = statistics.mean(times) / steps * full_steps
    sample = (f"first {args.cpu_restarts} restart(s) of the solve ({steps} Lanczos steps, "
              f"{statistics.mean(times):.1f} s), extrapolated to the {full_steps} Lanczos steps of a full solve")
    line = {"impl": "reference", "metric": "time_to_all_residuals_le_1e-7", "value": value, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded power-law matrix and start vector)",
            "config": cross_config(args, int(csr[0][-1])),
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_b200_cross(args):
    import torch

    import slepc_b200 as S

    from slepc_b200.ranks import Ranks

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    ranks = Ranks("nccl", timeout_s=600)  # replicas: barrier and max over ranks, no data-path collective
    barrier, max_over_ranks = ranks.barrier, ranks.max

    m, n = args.rows, args.cols
    csr, v0 = cross_workload(args)
    nnz = int(csr[0][-1])
    dt = np.float32 if args.svd_dtype == "f32" else np.float64
    vals = csr[2].astype(dt)
    A = S.Mat().createAIJ((csr[0], csr[1], vals), size=(m, n), dtype=dt)
    E = S.SVD().create()
    E.setOperators(A)
    E.setDimensions(args.nsv, args.svd_ncv)
    E.setTolerances(SVD_TOL)
    E.setInitialSpace(v0)

    def step():
        E.solve()
        E.getVectorPointers(0)  # SVDComputeVectors: U = A V, orthogonalised

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = S.kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = S.kernel_launch_count() - launches0
    ms_per_step = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    nconv = E.getConverged()
    reason = E.getConvergedReason()
    errs = [E.computeError(i) for i in range(min(nconv, args.nsv))]
    stats = E.getStats()

    E.setTiming(True)
    step()
    tstats = E.getStats()
    E.setTiming(False)
    peak, peak_kind = measured_peaks()
    vb = 4 if dt == np.float32 else 8
    # one application of A^T A: both CSR operands once, x and w read once and written once
    op_bytes = 2 * nnz * (vb + 4) + (m + 1 + n + 1) * 4 + 2 * (m + n) * 8
    spmv_gbs = (op_bytes * tstats["lanczos_steps"] / (tstats["ms_spmv"] * 1e-3) / 1e9
                if tstats["ms_spmv"] > 0 else None)
    gs_gbs = tstats["gs_bytes"] / (tstats["ms_orth"] * 1e-3) / 1e9 if tstats["ms_orth"] > 0 else None

    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_csr = (pin(csr[0]), pin(csr[1]), pin(vals))
    h_v0 = pin(v0)
    barrier()
    t0 = time.perf_counter()
    e2e_last = None
    for _ in range(args.steps):
        e2e_last = S.svd_solve_aij_host(h_csr, (m, n), h_v0, args.nsv, args.svd_ncv, tol=SVD_TOL, dtype=dt)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    h2d = csr[0].nbytes + csr[1].nbytes + vals.nbytes + v0.nbytes
    d2h = e2e_last["nconv"] * ((m + n) * 8 + 16)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t, r = cross_cpu_sample(csr, v0, args, threads)
        value = t / r.lanczos_steps * stats["lanczos_steps"]
        cpu = {"value": value, "unit": "s", "cores": threads, "kind": "port",
               "sample": (f"first {args.cpu_restarts} restart(s) of the same solve on {threads} host threads "
                          f"({r.lanczos_steps} Lanczos steps in {t:.1f} s), extrapolated to the "
                          f"{stats['lanczos_steps']} Lanczos steps of the full GPU solve")}
    if rank == 0:
        line = {"metric": "time_to_all_residuals_le_1e-7", "value": ms_per_step / 1e3, "unit": "s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded power-law matrix, seeded N(0,1) start vector)",
                "config": cross_config(args, nnz, {
                    "restarts": stats["restarts"], "lanczos_steps": stats["lanczos_steps"],
                    "column_visits": stats["column_visits"], "nconv": nconv, "reason": reason,
                    "max_rel_error": max(errs) if errs else None}),
                "roofline": {"kernel": "cross operator A^T A (warp-tile SpMV of A, segmented SpMV of A^T)",
                             "bound": "hbm", "achieved": spmv_gbs, "peak": peak, "unit": "GB/s",
                             "frac": (spmv_gbs / peak) if spmv_gbs else None, "peak_kind": peak_kind,
                             "traffic": None, "gs_achieved": gs_gbs,
                             "share_orth": tstats["ms_orth"] / tstats["ms_total"] if tstats["ms_total"] else None,
                             "share_spmv": tstats["ms_spmv"] / tstats["ms_total"] if tstats["ms_total"] else None,
                             "share_restart": tstats["ms_restart"] / tstats["ms_total"] if tstats["ms_total"] else None},
                "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(launches),
                "clocks": clk,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    E.destroy()
    A.destroy()
    ranks.close()
    return 0


# ------------------------------------------------------------------ batched workload
def batched_workload(args):
    ns = P.batch_sizes(args.nprob, 0)
    B = P.knn_batch(ns, 8, 0)
    v0 = np.concatenate([P.start_vector(int(n), p) for p, n in enumerate(ns)])
    return B, v0


def batched_config(args, B, extra=None):
    d = {"workload": f"{args.nprob} independent symmetric eigenproblems, n ~ U[500, 20000], each 2I - L_norm of a "
                     "symmetrised 8-NN graph of uniform points in the unit square, FP64 CSR, nev=8 largest real, "
                     "ncv=24, tol=1e-8, one persistent launch under a captured CUDA graph"
                     + (" (mixed: FP32-basis phase to 1e-6, then the FP64 solve from the phase-1 Ritz vectors, "
                        "three launches in one graph)" if args.precision == "mixed" else ""),
         "nprob": args.nprob, "rows": int(B.ns.sum()), "nnz": int(B.vals.size), "nev": 8, "ncv": 24, "tol": 1e-8,
         "start_vector": "N(0,1), seed = problem index",
         "l2": "inputs larger than L2: CSR %.1f GB, bases %.1f GB (L2 = 126 MB)"
               % (B.vals.size * 12 / 1e9, B.ns.sum() * 25 * 8 / 1e9),
         "parallelism": "replicas" if args.gpus > 1 else "single GPU"}
    if extra:
        d.update(extra)
    return d


def batched_cpu_sample(B, v0, args, threads, idx):
    import oracle

    sub_ns = B.ns[idx]
    rp, ci, va, vv = [], [], [], []
    for p in idx:
        r, c, v = B.problem(int(p))
        rp.append(r)
        ci.append(c)
        va.append(v)
        vv.append(v0[B.row_off[p]:B.row_off[p + 1]])
    t0 = time.perf_counter()
    ev, info = oracle.eps_solve_batch(sub_ns, np.concatenate(rp), np.concatenate(ci), np.concatenate(va),
                                      np.concatenate(vv), 8, 24, 1e-8, oracle.LARGEST_REAL, threads=threads)
    return time.perf_counter() - t0, info


def batched_sample_index(args, B):
    step = max(1, args.nprob // max(1, args.cpu_sample))
    return np.arange(0, args.nprob, step)[:args.cpu_sample]


class BatchShard:
    """The problems `idx` of a batch that one rank solves, with their start vectors."""

    def __init__(self, B, v0, idx):
        self.idx = list(idx)
        self.B = B.subset(self.idx) if B is not None else None
        self.v0 = B.rows_of(v0, self.idx) if (B is not None and v0 is not None) else None


def batched_shard(B, v0, rank, world):
    """Rank `rank` of `world` takes the contiguous range ranks.shard gives it (the whole batch at world 1)."""
    from slepc_b200.ranks import shard

    idx = shard(B.nprob, rank, world)
    if world == 1:
        s = BatchShard(None, None, idx)
        s.B, s.v0 = B, v0
        return s
    return BatchShard(B, v0, idx)


def run_reference_batched(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    B, v0 = batched_workload(args)
    threads = os.cpu_count() or 1
    idx = batched_sample_index(args, B)
    w_all = float(np.sum(B.ns.astype(np.float64) ** 2))
    w_s = float(np.sum(B.ns[idx].astype(np.float64) ** 2))
    for _ in range(args.warmup):
        batched_cpu_sample(B, v0, args, threads, idx)
    times = [batched_cpu_sample(B, v0, args, threads, idx)[0] for _ in range(args.steps)]
    value = statistics.mean(times) * w_all / w_s
    sample = (f"every {args.nprob // len(idx)}th problem ({len(idx)} problems, {statistics.mean(times):.1f} s on "
              f"{threads} threads, one problem per thread), extrapolated by the sum of n^2 (restarts grow with n)")
    line = {"impl": "reference", "metric": "time_to_all_residuals_le_1e-8", "value": value, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded k-NN graphs and start vectors)",
            "config": batched_config(args, B),
            "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_b200_batched(args):
    import torch

    import slepc_b200 as S

    from slepc_b200.ranks import Ranks, shard

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    ranks = Ranks("nccl", timeout_s=600)  # barrier, max and sum over ranks, no data-path collective
    barrier, max_over_ranks = ranks.barrier, ranks.max

    B_all, v0_all = batched_workload(args)
    # the problems are independent: each rank solves its contiguous share of the batch
    part = batched_shard(B_all, v0_all, rank, world)
    B, v0 = part.B, part.v0

    def make():
        E = S.BatchEPS().create(B.ns, B.rowptr, B.colind, B.vals)
        E.setDimensions(8, 24)
        E.setTolerances(1e-8)
        E.setWhichEigenpairs(S.LARGEST_REAL)
        E.setInitialVectors(v0)
        if args.precision == "mixed":
            E.setPrecision(S.EPS.Precision.MIXED, 1e-6)
        return E

    E = make()
    threads = E.autotune()
    for _ in range(args.warmup):
        E.solve()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = S.kernel_launch_count()
    dev_ms = []
    for _ in range(args.steps):
        E.solve()  # one graph replay; device time from CUDA events around it
        dev_ms.append(E.getAll()[2])
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = S.kernel_launch_count() - launches0
    ms_per_step = max_over_ranks(statistics.mean(dev_ms))
    ev, info, _ = E.getAll()
    bytes_moved = ranks.sum(E.getBytes())  # every rank's problems, over the slowest rank's time
    all_converged = ranks.sum(float(np.all(info[:, 2] == 1))) == world
    max_restarts = max_over_ranks(int(info[:, 1].max()) if len(info) else 0)
    lanczos_total = ranks.sum(int(info[:, 3].sum()))
    launches = int(ranks.sum(launches))
    peak, peak_kind = measured_peaks()
    achieved = bytes_moved / (ms_per_step * 1e-3) / 1e9

    # end to end: host CSR and start vectors in, eigenvalues out, through the public API
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        E2 = make()
        E2.setThreads(threads)
        E2.solve()
        ev2, info2, _ = E2.getAll()
        E2.destroy()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    h2d = ranks.sum(B.rowptr.nbytes + B.colind.nbytes + B.vals.nbytes + v0.nbytes + B.ns.nbytes)
    d2h = ranks.sum(ev2.nbytes + info2.nbytes)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ncpu = os.cpu_count() or 1
        idx = batched_sample_index(args, B)
        t, oinfo = batched_cpu_sample(B, v0, args, ncpu, idx)
        w = (B.ns.astype(np.float64) * info[:, 3]).sum() / (B.ns[idx].astype(np.float64) * info[idx, 3]).sum()
        cpu = {"value": t * w, "unit": "s", "cores": ncpu, "kind": "port",
               "sample": (f"{len(idx)} of the {args.nprob} problems (every {args.nprob // len(idx)}th) on {ncpu} "
                          f"threads, one problem per thread, {t:.1f} s, extrapolated by the sum over problems of "
                          f"n x Lanczos steps of the GPU solve")}
    if rank == 0:
        line = {"metric": "time_to_all_residuals_le_1e-8", "value": ms_per_step / 1e3, "unit": "s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": False, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32 basis then f64" if args.precision == "mixed" else "f64",
                "data": "synthetic (seeded k-NN graphs, seeded N(0,1) start vectors)",
                "config": batched_config(args, B_all, {
                    "threads_per_problem": threads, "all_converged": bool(all_converged),
                    "max_restarts": int(max_restarts), "lanczos_steps": int(lanczos_total),
                    "problems_per_rank": [len(shard(B_all.nprob, r, world)) for r in range(world)]}),
                "roofline": {"kernel": "batched_ks_kernel (whole Krylov-Schur per CTA)", "bound": "hbm",
                             "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "peak_kind": peak_kind, "traffic": None,
                             "algorithmic_bytes_per_step": bytes_moved},
                "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(launches),
                "clocks": clk,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    E.destroy()
    ranks.close()
    return 0


# ------------------------------------------------------------------ learned warm start workload
EVAL_SEED0 = 100000


def learned_config(args, extra=None):
    held = args.eval_fields * args.steps
    reduced = ""
    if args.learn_grid == 512 and (args.train_fields < 2000 or held < 200):
        reduced = (f"the 512^2 / 2000 training / 200 held-out configuration reduced to {args.train_fields} training "
                   f"and {held} held-out fields: ")
    orth = {"gs": "Gram-Schmidt", "chol": "Cholesky"}[args.learn_orthog]
    d = {"workload": (reduced + f"{args.learn_nev} smallest eigenpairs of -div(kappa grad u) on a {args.learn_grid}^2 "
                      "grid (5-point FV, kappa = exp(GRF), variance 1, correlation length U[0.05, 0.2]) by LOBPCG "
                      f"(Jacobi, block {args.learn_nev}, {orth} block orthogonalization, tol 1e-8) on {held} held-out "
                      f"fields ({args.eval_fields} per step; {args.warmup * args.eval_fields} more in the warm-up steps), "
                      "started from the "
                      "neural operator's block; the network "
                      f"(width 32, {args.learn_modes} x {args.learn_modes} modes, 4 layers, tensor-core GEMMs) trained "
                      f"on the plain solver's eigenvectors of {args.train_fields} fields, {args.epochs} epochs"),
         "grid": args.learn_grid, "nev": args.learn_nev, "train_fields": args.train_fields,
         "eval_fields": held, "eval_fields_per_step": args.eval_fields, "epochs": args.epochs, "tol": 1e-8,
         "orthog_block": args.learn_orthog,
         "l2": "fields of %d x %d cells; every solve is a separate operator" % (args.learn_grid, args.learn_grid),
         "parallelism": "single GPU"}
    if extra:
        d.update(extra)
    return d


def run_b200_learned(args):
    import torch

    import slepc_b200 as S
    from slepc_b200 import learned as LN

    from slepc_b200.ranks import Ranks

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    ranks = Ranks("nccl", timeout_s=3600)  # replicas: each rank trains and evaluates its own copy
    N, nev = args.learn_grid, args.learn_nev
    t0 = time.perf_counter()
    ob = S.BV.OrthogBlockType.CHOL if args.learn_orthog == "chol" else None
    F, T, its_train = LN.dataset(S, N, range(args.train_fields), nev, orthog_block=ob)
    t_data = time.perf_counter() - t0
    dims = (N, 32, args.learn_modes, 4, 64, nev)
    op = S.NeuralOperator().create(*dims)
    op.setParams(LN.init_params(*dims, seed=0))
    Fd, Td = torch.from_numpy(F).cuda(), torch.from_numpy(T).cuda()
    t0 = time.perf_counter()
    hist = LN.train(op, Fd, Td, epochs=args.epochs, batch=8, lr=2e-3, lr_final=2e-4)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    # held-out fields: every step (warm-up and timed) solves its own eval_fields fields, and each rank
    # its own range of seeds (weak scaling)
    E = args.eval_fields
    span = (args.warmup + args.steps) * E
    base = EVAL_SEED0 + rank * span

    def fields(step_index):
        seeds_i = list(range(base + step_index * E, base + (step_index + 1) * E))
        probs_i = [P.diffusion_problem(N, sd) for sd in seeds_i]
        feats_i = torch.from_numpy(np.stack([LN.features(k) for _, k, _ in probs_i])).cuda()
        return seeds_i, probs_i, feats_i

    warm = [fields(i) for i in range(args.warmup)]
    timed = [fields(args.warmup + i) for i in range(args.steps)]
    seeds = [sd for sd_i, _, _ in timed for sd in sd_i]

    def step(batch, learned):
        _, probs_i, feats_i = batch
        blocks = LN.predict(op, feats_i) if learned else None
        out = []
        for i, (csr, _, _) in enumerate(probs_i):
            X0 = blocks[i].T.astype(np.float64) if learned else None
            out.append(LN.solve_lowest(S, csr, nev, X0=X0, orthog_block=ob))
        return out

    for bt in warm:
        step(bt, True)
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = S.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    res_l = []
    for bt in timed:
        res_l += step(bt, True)
    ev1.record()
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = S.kernel_launch_count() - launches0
    ms_step = ranks.max(ev0.elapsed_time(ev1) / args.steps)
    # the same timed fields from the seeded random block (the fallback)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res_r = []
    for bt in timed:
        res_r += step(bt, False)
    e1.record()
    torch.cuda.synchronize()
    ms_random = ranks.max(e0.elapsed_time(e1) / args.steps)
    # end to end on the first e2e_steps timed steps: host fields in, host eigenpairs out (features up,
    # network, block down, solve, pairs down)
    ne2e = max(1, min(args.e2e_steps or args.steps, args.steps))
    t0 = time.perf_counter()
    for _, probs_i, _ in timed[:ne2e]:
        hf = torch.from_numpy(np.stack([LN.features(k) for _, k, _ in probs_i])).pin_memory()
        blocks = LN.predict(op, hf.cuda(non_blocking=True))
        for i, (csr, _, _) in enumerate(probs_i):
            LN.solve_lowest(S, csr, nev, X0=blocks[i].T.astype(np.float64), orthog_block=ob)
    e2e_s = ranks.max((time.perf_counter() - t0) / ne2e)
    preds = np.concatenate([LN.predict(op, f) for _, _, f in timed])
    captured = [LN.captured(r["X"], b.T.astype(np.float64)) for r, b in zip(res_r, preds)]
    its_l = [r["its"] for r in res_l]
    its_r = [r["its"] for r in res_r]
    good = lambda rs: all(r["nconv"] >= nev and r["max_error"] <= 1e-8 for r in rs)
    ok = good(res_l + res_r)
    probs = timed[0][1]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        csr0 = probs[0][0]
        oob = oracle.ORTHOG_BLOCK_CHOL if args.learn_orthog == "chol" else oracle.ORTHOG_BLOCK_GS
        t0 = time.perf_counter()
        r = oracle.lobpcg(P.to_scipy(csr0), nev, tol=1e-8, max_it=args.cpu_max_it or 100000, orthog_block=oob)
        tc = time.perf_counter() - t0
        if args.cpu_max_it:
            its_gpu = res_r[0]["its"]
            cpu = {"value": tc / max(r.its, 1) * its_gpu, "unit": "s per field", "cores": threads, "kind": "port",
                   "sample": f"oracle LOBPCG from the random block on held-out field {seeds[0]}: {r.its} iterations "
                             f"in {tc:.1f} s, scaled to the {its_gpu} iterations of the GPU solve from the random "
                             "block"}
        else:
            cpu = {"value": tc, "unit": "s per field", "cores": threads, "kind": "port",
                   "sample": f"oracle LOBPCG from the random block on held-out field {seeds[0]} ({r.its} iterations)"}
    if rank == 0:
        n = E
        wins = int(sum(1 for a_, b_ in zip(its_l, its_r) if a_ < b_))
        line = {"metric": "time_to_all_residuals_le_1e-8_per_field", "value": ms_step / 1e3 / n, "unit": "s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64 solve, f32 network",
                "data": "synthetic (seeded Gaussian random fields)",
                "config": learned_config(args, {"dataset_seconds": t_data, "train_seconds": t_train,
                                                "final_train_loss": hist[-1],
                                                "mean_train_solve_iterations": float(np.mean(its_train))}),
                "learned_vs_random": {"s_per_field_random": ms_random / 1e3 / n, "speedup": ms_random / ms_step,
                                      "mean_iterations_learned": float(np.mean(its_l)),
                                      "mean_iterations_random": float(np.mean(its_r)),
                                      "iterations_learned": its_l, "iterations_random": its_r,
                                      "fields_with_fewer_iterations": wins, "fields": len(its_l),
                                      "max_error_learned": [r["max_error"] for r in res_l],
                                      "max_error_random": [r["max_error"] for r in res_r],
                                      "nconv_learned": [r["nconv"] for r in res_l],
                                      "nconv_random": [r["nconv"] for r in res_r],
                                      "reason_learned": [r["reason"] for r in res_l],
                                      "reason_random": [r["reason"] for r in res_r],
                                      "held_out_seeds": seeds,
                                      "mean_captured_subspace": float(np.mean(captured)),
                                      "all_pairs_converged_to_1e-8": ok,
                                      "learned_all_pairs_le_1e-8": good(res_l),
                                      "random_all_pairs_le_1e-8": good(res_r)},
                "roofline": None,
                "e2e": {"value": e2e_s / n, "unit": "s", "h2d_bytes_per_step": int(n * 3 * N * N * 4),
                        "d2h_bytes_per_step": int(n * nev * N * N * 12), "steps": ne2e},
                "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": cpu}
        print(json.dumps(line))
    op.destroy()
    ranks.close()
    return 0


def main():
    args = parse()
    if args.workload == "learned":
        if args.impl == "reference":
            if dist_env()[0] != 0:
                return 0
            print(json.dumps({"impl": "reference", "unavailable": "the learned workload has no reference arm: SLEPc "
                              "has no learned start; its CPU baseline (oracle LOBPCG) is in the b200 line"}))
            return 0
        return run_b200_learned(args)
    if args.workload == "batched":
        if args.impl == "reference":
            return run_reference_batched(args)
        return run_b200_batched(args)
    if args.workload == "cross":
        if args.impl == "reference":
            return run_reference_cross(args)
        return run_b200_cross(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
