"""The N > 1 host path on CPU: world-size-2 process groups on gloo.

bench.py runs one replica per GPU; what the ranks share is a barrier on both
sides of the timed region, the maximum of each rank's time and the rule that
only rank 0 reports (and only rank 0 runs the CPU reference arm).  The same
`Ranks` object runs here on the gloo backend.
"""
import contextlib
import io
import os
import socket
import sys
import tempfile

import pytest

from slepc_b200.ranks import Ranks, env, shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, plan):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r = Ranks("gloo", timeout_s=60)
    assert (r.rank, r.local_rank, r.world) == (rank, rank, world)
    r.barrier()
    got = [r.max(x) for x in plan[rank]]  # every rank takes the same collectives in the same order
    r.barrier()
    r.close()
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(" ".join(repr(v) for v in got))


def _batch_worker(rank, world, port, out_dir, nprob):
    """One rank of the sharded batched workload, with the oracle's batch solver standing in for the
    GPU launch: the rank solves only its share of the problems and reports a sum over ranks."""
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    import oracle
    from slepc_b200 import problems as P

    r = Ranks("gloo", timeout_s=60)
    ns = P.batch_sizes(nprob, 3, lo=60, hi=200)
    B = P.knn_batch(ns, 8, 3)
    v0 = np.concatenate([P.start_vector(int(n), p) for p, n in enumerate(ns)])
    part = bench.batched_shard(B, v0, rank, world)
    ev, info = oracle.eps_solve_batch(part.B.ns, part.B.rowptr, part.B.colind, part.B.vals, part.v0, 4, 12, 1e-8,
                                      oracle.LARGEST_REAL, threads=1)
    total_rows = r.sum(int(part.B.ns.sum()))
    r.close()
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), idx=np.array(part.idx), ev=ev, info=info,
             total_rows=total_rows)


def test_sharded_batch_union_equals_single_rank():
    """The batched workload split over two gloo ranks: every problem is solved by exactly one rank
    and the union of their results equals the one-rank run of the whole batch."""
    import numpy as np
    import torch.multiprocessing as mp

    import oracle
    from slepc_b200 import problems as P

    nprob = 7
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_batch_worker, args=(2, _free_port(), d, nprob), nprocs=2, join=True,
                           start_method="spawn")
        parts = [np.load(os.path.join(d, f"rank{r}.npz")) for r in range(2)]
    idx = np.concatenate([p["idx"] for p in parts])
    assert sorted(idx.tolist()) == list(range(nprob)) and len(idx) == nprob
    ns = P.batch_sizes(nprob, 3, lo=60, hi=200)
    assert all(float(p["total_rows"]) == float(ns.sum()) for p in parts)
    B = P.knn_batch(ns, 8, 3)
    v0 = np.concatenate([P.start_vector(int(n), p) for p, n in enumerate(ns)])
    ev, info = oracle.eps_solve_batch(B.ns, B.rowptr, B.colind, B.vals, v0, 4, 12, 1e-8, oracle.LARGEST_REAL,
                                      threads=1)
    got_ev = np.concatenate([p["ev"] for p in parts])
    got_info = np.concatenate([p["info"] for p in parts])
    np.testing.assert_array_equal(got_ev, ev[idx])
    np.testing.assert_array_equal(got_info, info[idx])


def test_shard_partitions_every_unit_once():
    for count in (0, 1, 5, 8, 4096, 4097):
        for world in (1, 2, 3, 8):
            parts = [shard(count, r, world) for r in range(world)]
            units = [u for p in parts for u in p]
            assert units == list(range(count))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def test_single_rank_is_local(monkeypatch):
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    assert env() == (0, 0, 1)
    r = Ranks("gloo")
    assert r.dist is None
    r.barrier()
    assert r.max(2.5) == 2.5
    r.close()


def test_world_size_2_barrier_and_max_over_ranks():
    import torch.multiprocessing as mp

    plan = {0: [3.0, -1.0, 7.25], 1: [5.5, -4.0, 0.0]}
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), d, plan), nprocs=2, join=True, start_method="spawn")
        for rank in range(2):
            with open(os.path.join(d, f"rank{rank}.txt")) as f:
                got = [float(v) for v in f.read().split()]
            assert got == [5.5, -1.0, 7.25]


@pytest.mark.parametrize("workload", ["laplacian3d", "batched", "cross", "learned"])
def test_reference_arm_runs_on_rank_0_only(monkeypatch, workload):
    """Under torchrun the reference arm's other ranks exit 0 without work or output."""
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--workload", workload, "--gpus", "2"])
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.main() == 0
    assert buf.getvalue() == ""
