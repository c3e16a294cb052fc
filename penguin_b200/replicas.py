"""Replicas across the GPUs of one node.

A Godunov step of one disk has no exchange with any other disk: the
reference runs one disk per process and never splits it (main.cu:165-360
allocates the whole grid on one device).  So several GPUs run independent
replicas, one process per GPU, each stepping its own seeded disk, and the
data path carries no collective.  The process group is used for timing only:
a barrier on both sides of the timed region and the maximum of the ranks'
device times, from which the whole-job rate is the units every rank
processed divided by that maximum.

An ensemble of disks shards the same way, by whole disks: ``partition``
splits the disks across the ranks by their cell counts, each rank steps its
share as one ensemble, and ``gather`` brings the results to rank 0 at the end.

The launcher (torchrun) sets WORLD_SIZE, RANK and LOCAL_RANK and the
MASTER_ADDR / MASTER_PORT rendezvous.  The backend is NCCL on the GPUs and
gloo on the host cores; every rank takes the same collective calls in the same
order.
"""
from __future__ import annotations

import datetime
import os
from typing import Callable, Mapping


class Replicas:
    """The ranks of one job.  With WORLD_SIZE 1 (or unset) no process group is
    created and every call is local."""

    def __init__(self, backend: str | None = None, timeout_s: float = 120.0,
                 env: Mapping[str, str] | None = None):
        env = os.environ if env is None else env
        self.world = int(env.get("WORLD_SIZE", "1"))
        self.rank = int(env.get("RANK", "0"))
        self.local = int(env.get("LOCAL_RANK", "0"))
        if self.world < 1 or not 0 <= self.rank < self.world or self.local < 0:
            raise ValueError(f"bad rank layout: world {self.world}, rank {self.rank}, local {self.local}")
        import torch

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        self.backend = backend
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if backend == "nccl":
            torch.cuda.set_device(self.local)  # this process's GPU, before the group binds one
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            if dist.get_world_size() != self.world or dist.get_rank() != self.rank:
                raise RuntimeError("process group disagrees with WORLD_SIZE / RANK")
            self.dist = dist

    @property
    def printer(self) -> bool:
        """Rank 0 alone reports for the job."""
        return self.rank == 0

    def seed(self, base: int) -> int:
        """Each replica steps its own disk: the seed of its initial noise."""
        return base + self.rank

    def barrier(self, sync: Callable[[], None] | None = None) -> None:
        """All ranks meet, then ``sync`` (the local device synchronise) runs."""
        if self.dist is not None:
            self.dist.barrier()
        if sync is not None:
            sync()

    def max_over_ranks(self, x: float) -> float:
        """The largest of the ranks' values (each rank passes its own)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def job_rate(self, units_per_rank: float, ms: float) -> float:
        """Whole-job throughput: every rank processed ``units_per_rank`` in at
        most ``ms`` (the max over ranks)."""
        if ms <= 0.0:
            raise ValueError("non-positive time")
        return units_per_rank * self.world / (ms / 1000.0)

    def share(self, weights) -> list[int]:
        """The indices of the independent units (ensemble disks) this rank runs."""
        return partition(weights, self.world)[self.rank]

    def gather(self, obj):
        """Every rank's ``obj`` in rank order on rank 0 (None on the others): the
        final host-side gather of a partitioned ensemble's results."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world if self.printer else None
        self.dist.gather_object(obj, out, dst=0)
        return out

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def partition(weights, world: int) -> list[list[int]]:
    """Whole units across ``world`` ranks, balanced by weight (cells x steps):
    the heaviest unit first, each to the rank with the least weight so far
    (ties to the lower rank).  Deterministic, so every rank computes the same
    split without communication.  Each rank's list is in ascending index
    order."""
    if world < 1:
        raise ValueError("world must be positive")
    w = [float(x) for x in weights]
    if any(not x >= 0.0 for x in w):
        raise ValueError("weights must be non-negative")
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(w)), key=lambda i: (-w[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += w[k]
    return [sorted(p) for p in parts]
