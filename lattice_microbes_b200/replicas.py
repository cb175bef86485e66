"""Replica runs on several GPUs: one process per GPU over torch.distributed.

The MPD-RDME path shards across replicates with no data exchange, as
ReplicateRunner threads run one solver per replicate (core/ReplicateRunner.cpp:
84-166): rank r runs replicate r -- its own seed, composed from the seed top
and the replicate number as MpdRdmeSolver::initialize does
(MpdRdmeSolver.cu:112-123), and its own lattice -- on its own GPU.  The only
collective steps are the barriers that bracket a timed region and the
max-over-ranks reduction of its time; every rank takes them in the same order.
"""
import datetime
import os

from .solver import compose_seed


class Ranks:
    """The process's place in a torch.distributed.run launch (WORLD_SIZE,
    RANK, LOCAL_RANK; a single process when they are absent)."""

    def __init__(self, environ=None):
        e = os.environ if environ is None else environ
        self.world = int(e.get("WORLD_SIZE", "1"))
        self.rank = int(e.get("RANK", "0"))
        self.local = int(e.get("LOCAL_RANK", "0"))
        self.group = False

    @property
    def leader(self):
        """Rank 0: the one that prints results."""
        return self.rank == 0

    def init(self, backend="nccl", timeout_s=120):
        """Joins the process group (N > 1 only) with a short timeout, so that
        ranks waiting on a rank that died end with an error."""
        if self.world > 1 and not self.group:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.group = True
        return self

    def seed(self, seed_top):
        """The seed of this rank's replicate."""
        return compose_seed(seed_top, self.rank)

    def barrier(self):
        if self.group:
            import torch.distributed as dist
            dist.barrier()

    def max(self, value, device="cpu"):
        """The largest `value` over the ranks (the slowest rank's time)."""
        if not self.group:
            return float(value)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def finish(self):
        if self.group:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
            self.group = False


def aggregate_rate(units_per_rank, slowest_ms, world):
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time (weak scaling: each rank processes the same amount)."""
    return units_per_rank * world / (slowest_ms / 1e3)
