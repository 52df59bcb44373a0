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
