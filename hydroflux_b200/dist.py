"""One process per GPU: ranks, timing reductions and scenario sharding.

The solver's units of parallel work across GPUs are independent: a grid fits
one B200, so several GPUs run replicas, or split an ensemble / a request
stream by scenario. No step needs a data-path collective; torch.distributed
only provides the barrier around timed regions, the max over ranks of a time
and the gathering of per-rank results on rank 0 (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import datetime
import heapq
import os
from typing import Any, List, Optional, Sequence


def lpt_shards(weights: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time-first partition of units with the given
    weights (e.g. cell counts) over `world` ranks: units in decreasing
    weight, each to the currently lightest rank (ties to the lower rank).
    Deterministic; every unit goes to exactly one rank; the heaviest rank
    carries at most 4/3 of the optimum (Graham's bound). Indices within a
    shard keep their original order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(s) for s in shards]


class Dist:
    """RANK / LOCAL_RANK / WORLD_SIZE from the environment (torchrun). With
    world > 1 a process group is created: NCCL with the GPU of LOCAL_RANK, or
    gloo when use_gpu is False. Its timeout is short so that ranks waiting on
    a rank that died end with an error instead of hanging."""

    def __init__(self, use_gpu: bool = True, timeout_s: float = 600.0,
                 backend: Optional[str] = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        self.use_gpu = use_gpu
        if self.world > 1:
            import torch
            import torch.distributed as dist
            be = backend or ("nccl" if use_gpu else "gloo")
            kw = {}
            if be == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(be, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.backend = be
            self.pg = True

    def _device(self):
        import torch
        return torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")

    def barrier(self) -> None:
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        """Max over ranks (e.g. of a timed region: the job ends with its
        slowest rank)."""
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self._device())
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self._device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj: Any) -> Optional[List[Any]]:
        """Every rank's object on rank 0 (None elsewhere)."""
        if not self.pg:
            return [obj]
        import torch.distributed as dist
        out = [None] * self.world if self.rank == 0 else None
        dist.gather_object(obj, out, dst=0)
        return out

    def shard(self, weights: Sequence[float]) -> List[int]:
        """This rank's unit indices under lpt_shards."""
        return lpt_shards(weights, self.world)[self.rank]

    def close(self) -> None:
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()
            self.pg = False
