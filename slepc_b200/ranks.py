"""One process per GPU for replica runs.

The eigensolver path is run as independent replicas, one per GPU: every rank
solves its own copy of the problem, or its own share of a batch of independent
problems (``shard``), and no data-path collective exists.  What the ranks share is host plumbing: the
torchrun environment, a barrier on both sides of a timed region and the maximum
of a host number (a per-rank time) over the ranks, taken on rank 0's report.

``Ranks(backend="nccl")`` is what a GPU run uses; ``backend="gloo"`` runs the
same logic on CPU processes.  With WORLD_SIZE 1 no process group is created and
every call is local.
"""
import datetime
import os


def env():
    """(rank, local rank, world size) from the torchrun environment (0, 0, 1 without it)."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def shard(count, rank, world):
    """The contiguous range of `count` independent units that `rank` of `world` owns: the first
    count % world ranks take one unit more; every unit belongs to exactly one rank."""
    if count < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("invalid shard arguments")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


class Ranks:
    """The process group of a replica run (created only when WORLD_SIZE > 1)."""

    def __init__(self, backend="nccl", timeout_s=600):
        self.rank, self.local_rank, self.world = env()
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """The maximum of the host number x over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        """The sum of the host number x over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
