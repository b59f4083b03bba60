"""Replica parallelism over configurations.

The measurement path shards over gauge configurations only: every process
(one per GPU) measures whole configurations on its own device, and no
collective touches the data path.  The process group exists for three host
decisions: which configurations a rank owns, a barrier around timed regions,
and the maximum of the per-rank times (the job is as slow as its slowest
replica).  The reference instead splits one lattice over MPI ranks with halo
exchanges (modules/lnk/lnkcom.c); a whole configuration fits one B200.
"""
from __future__ import annotations

import datetime
import os
from typing import List, Sequence, TypeVar

T = TypeVar("T")


def env_ranks():
    """(rank, world, local_rank) from the torchrun environment; (0, 1, 0)
    for a plain process."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def config_numbers(first: int, last: int, step: int) -> List[int]:
    """The configuration numbers ms10 visits: first, first+step, ..., <= last
    (main/ms10.c:701)."""
    if step < 1:
        raise ValueError("step must be >= 1")
    return list(range(first, last + 1, step))


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin ownership: rank r measures items r, r+world, ...  Every
    item has exactly one owner, and the ranks' loads differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return list(items[rank::world])


class Replicas:
    """The replica group of this process.

    With world 1 no process group is created and every method is local.
    Otherwise `torch.distributed` is initialised from the environment with
    `backend` ("nccl" on GPUs, "gloo" on the CPU) and a short timeout, so a
    rank that died makes the others' next collective fail instead of hang.
    """

    def __init__(self, backend: str | None = None, timeout_s: float = 300.0):
        self.rank, self.world, self.local = env_ranks()
        self.dist = None
        self.backend = None
        self.device = self.local
        if self.world > 1:
            import torch
            import torch.distributed as dist
            ndev = torch.cuda.device_count() if torch.cuda.is_available() else 0
            if ndev:
                # more ranks than visible GPUs share them round-robin; NCCL
                # cannot hold two ranks of one group on one GPU, so such a
                # group talks over gloo (its collectives are host decisions only)
                self.device = self.local % ndev
            if backend is None:
                backend = "nccl" if 0 < ndev and self.world <= ndev else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.device)
            if not dist.is_initialized():
                dist.init_process_group(backend,
                                        timeout=datetime.timedelta(seconds=timeout_s))
            self.dist, self.backend = dist, backend

    def _device(self):
        return f"cuda:{self.device}" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        """Sum of x over the ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def owned(self, items: Sequence[T]) -> List[T]:
        return shard(items, self.rank, self.world)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
