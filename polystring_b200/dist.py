"""Rank plumbing for runs of one process per GPU (torchrun environment).

A single SCFT solve does not shard (a 3D FFT would need an all-to-all per
axis pass), so N > 1 runs are replicas of a solve, or shards of independent
units (string images, batch solves) with no exchange on the data path.  This
module holds what those runs share: process-group set-up with a short
timeout, barriers, reductions of timings over ranks (a multi-GPU time is the
maximum over ranks), and the partition of units over ranks.  The backend is
NCCL on GPUs; the same code runs on gloo for the CPU tests.
"""
import datetime
import os


class Ranks:
    def __init__(self, backend=None, timeout_s=120):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch.distributed as dist
            backend = backend or "nccl"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            if backend == "nccl":
                self.device = "cuda"

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def _reduce(self, x, op):
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def allmax(self, x):
        """maximum over ranks (the time of a multi-GPU step)"""
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def allsum(self, x):
        """sum over ranks (the units all ranks processed)"""
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def shard(n_units, rank, world):
    """Contiguous block of unit indices owned by `rank`: sizes differ by at
    most one, every unit is owned by exactly one rank, order is kept."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n_units, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def throughput(units_per_rank, seconds_per_rank, ranks):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return ranks.allsum(units_per_rank) / ranks.allmax(seconds_per_rank)
