"""Host side of running on several GPUs: one process per GPU, no data-path
collective.

A single scene does not shard in this design, so N ranks run N independent
replicas.  A batch of independent scenes shards by scene: `partition_scenes`
assigns scenes to ranks by particle count (longest processing time first),
and each rank advances its own `BatchIISPH`.  The only collectives are the
reductions of the measurement: the slowest rank's time and the total work.
"""

from __future__ import annotations

import datetime
import os


def partition_scenes(sizes, world: int) -> list[list[int]]:
    """Scene indices per rank.  Greedy longest-processing-time: scenes in
    descending size (ties by index) each go to the rank with the least work so
    far (ties to the lower rank).  Every scene lands on exactly one rank; each
    rank's list is in ascending scene order; the result depends only on
    (sizes, world)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(p) for p in parts]


def env_rank() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, device=None, timeout_s: float = 120.0):
    """Join the process group described by the environment (MASTER_ADDR,
    MASTER_PORT, RANK, WORLD_SIZE); returns torch.distributed, or None for a
    single process."""
    rank, world, _ = env_rank()
    if world <= 1:
        return None
    import torch.distributed as dist

    kw = {"device_id": device} if (device is not None and backend == "nccl") else {}
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), rank=rank,
                            world_size=world, **kw)
    return dist


def _reduce(value: float, op_name: str, dist, device) -> float:
    import torch

    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The slowest rank's time (every rank gets it)."""
    return _reduce(value, "MAX", dist, device)


def sum_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Total work over ranks (every rank gets it)."""
    return _reduce(value, "SUM", dist, device)
