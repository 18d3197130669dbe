"""Independent replicas on the GPUs of one node: one process per GPU, no data-path collective.

The 1M-atom Lennard-Jones path does not shard without a halo exchange, so N GPUs run N
independent replicas (weak scaling): the process group carries only the barriers around a
timed region and the maximum of the ranks' times. Serving shards by replica: requests are
assigned to ranks by their atom-steps, so each rank's share of the work is about the same,
and each rank serves its share on its own GPU.
"""

from __future__ import annotations

import os
from datetime import timedelta

import torch
import torch.distributed as dist


class Ranks:
    """This process's place among the ranks (RANK, WORLD_SIZE, LOCAL_RANK from the launcher).

    With more than one rank it joins the process group (``backend`` "nccl" on GPUs, "gloo"
    on the host) with a short ``timeout``, so ranks that wait on a lost peer fail with an
    error instead of hanging.
    """

    def __init__(self, backend: str = "nccl", device: torch.device | None = None,
                 timeout_s: float = 300.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device if device is not None else torch.device("cpu")
        self.backend = backend
        self._joined = False
        if self.world > 1:
            kwargs = {"timeout": timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kwargs["device_id"] = self.device
            dist.init_process_group(backend, **kwargs)
            self._joined = True

    def barrier(self) -> None:
        if self._joined:
            dist.barrier()

    def max(self, value: float) -> float:
        """The largest ``value`` over the ranks (every rank gets it)."""
        if not self._joined:
            return float(value)
        where = self.device if self.backend == "nccl" else torch.device("cpu")
        tensor = torch.tensor([float(value)], dtype=torch.float64, device=where)
        dist.all_reduce(tensor, op=dist.ReduceOp.MAX)
        return float(tensor)

    def sum(self, value: float) -> float:
        """The sum of ``value`` over the ranks (every rank gets it)."""
        if not self._joined:
            return float(value)
        where = self.device if self.backend == "nccl" else torch.device("cpu")
        tensor = torch.tensor([float(value)], dtype=torch.float64, device=where)
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM)
        return float(tensor)

    def gather(self, rows: list) -> list:
        """Every rank's ``rows`` (picklable items), concatenated in rank order, on every rank.
        Host objects only: per-request results of a shard, not device data."""
        if not self._joined:
            return list(rows)
        parts: list = [None] * self.world
        dist.all_gather_object(parts, list(rows))
        return [row for part in parts for row in part]

    def close(self) -> None:
        if self._joined:
            dist.destroy_process_group()
            self._joined = False


def shard_requests(work: list[float], world: int) -> list[list[int]]:
    """Indices of the requests each rank serves, given each request's work (atom-steps).

    Largest first, each to the rank with the least work so far (ties to the lower rank): the
    same answer on every rank, every request exactly once, and no rank above the average by
    more than its largest request.
    """
    if world < 1:
        raise ValueError("world must be at least 1")
    loads = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for index in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        rank = min(range(world), key=lambda r: (loads[r], r))
        shards[rank].append(index)
        loads[rank] += work[index]
    return [sorted(shard) for shard in shards]


__all__ = ("Ranks", "shard_requests")
