"""Replicas: independent cases spread over ranks, one process a GPU, no data-path collective.

The delta-SPH step of one case runs on one GPU; what shards across GPUs are independent cases (a
batched parameter sweep, a stream of requests).  Each rank steps its own cases; the only traffic
between ranks is the bookkeeping below: the barrier that brackets a timed region, the maximum of
the ranks' device times, and the gathering of per-case results on rank 0.  The backend is NCCL on
GPUs (tensors on the rank's device) and gloo on CPU (the multi-process tests).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int

    @property
    def distributed(self) -> bool:
        return self.world > 1


def ranksFromEnvironment() -> Ranks:
    """RANK, WORLD_SIZE and LOCAL_RANK as torch.distributed.run sets them (one rank by default)."""
    return Ranks(int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')),
                 int(os.environ.get('LOCAL_RANK', '0')))


def initialize(ranks: Ranks, backend: str = 'nccl', timeoutSeconds: float = 300.0) -> None:
    """Join the process group (nothing for one rank); a short timeout ends a rank that waits for a
    peer that is gone with an error instead of a hang."""
    if not ranks.distributed:
        return
    import torch
    import torch.distributed as dist
    kwargs = {}
    if backend == 'nccl':
        kwargs['device_id'] = torch.device('cuda', ranks.local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeoutSeconds), rank=ranks.rank,
                            world_size=ranks.world, **kwargs)


def finalize(ranks: Ranks) -> None:
    if ranks.distributed:
        import torch.distributed as dist
        dist.destroy_process_group()


def shard(items, ranks: Ranks) -> list:
    """This rank's share of independent items: every world-th one from its rank, so that the
    shares differ in size by one at most and a seeded list splits the same way every time."""
    return list(items)[ranks.rank::ranks.world]


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == 'nccl':
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


def barrier(ranks: Ranks) -> None:
    if ranks.distributed:
        import torch.distributed as dist
        dist.barrier()


def maxOverRanks(value: float, ranks: Ranks) -> float:
    """The largest of the ranks' values (a timed region's device time: the job ends with its slowest
    rank)."""
    if not ranks.distributed:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sumOverRanks(value: float, ranks: Ranks) -> float:
    if not ranks.distributed:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gatherResults(results: list, ranks: Ranks) -> list | None:
    """Every rank's list of per-case results, concatenated in rank order, on rank 0 (None on the
    others)."""
    if not ranks.distributed:
        return list(results)
    import torch.distributed as dist
    gathered = [None] * ranks.world if ranks.rank == 0 else None
    dist.gather_object(list(results), gathered, dst=0)
    if ranks.rank != 0:
        return None
    return [item for part in gathered for item in part]
