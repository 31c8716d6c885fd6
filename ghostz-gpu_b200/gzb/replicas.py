"""Multi-GPU plumbing of the benchmark: one process per GPU, each holding
its own copy of the chunk and searching either the whole query set (a
replica, as the reference's -g threads replicate the work) or its slice of
the queries (gzb.shards.query_range).  Queries are independent of each
other, so nothing on this path is exchanged between devices: the process
group carries only the barrier around the timed region, the slowest rank's
time and the ranks' query counts."""
import os
from datetime import timedelta


class Replicas:
    """Rank, world size and the collectives the timed region needs.  With
    WORLD_SIZE unset or 1 nothing is initialised and every call is local."""

    def __init__(self, backend="nccl", timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist
            self.device = "cuda" if backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, values):
        """Element-wise maximum over ranks of a list of floats."""
        if self.dist is None:
            return [float(v) for v in values]
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return [float(v) for v in t.cpu()]

    def throughput(self, units_per_rank, steps, max_ms):
        """Whole-job rate: every rank's units over the slowest rank's time."""
        return self.world * units_per_rank * steps / (max_ms / 1e3)

    def sum(self, values):
        """Element-wise sum over ranks of a list of numbers."""
        if self.dist is None:
            return [float(v) for v in values]
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return [float(v) for v in t.cpu()]

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
