"""One process per GPU, independent replicas: the plumbing bench.py and sweep
runs use under torchrun.  The solver path has no data exchange between GPUs
(a 128^2 x 32 grid is 4 MiB; sweep members are independent), so the process
group carries only the start/stop barrier and the max / sum of per-rank
timings and counts.  Backend "nccl" on GPUs, "gloo" for the CPU tests."""
from __future__ import annotations

import datetime
import os
from typing import Sequence, TypeVar

T = TypeVar("T")


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(ws: int, local: int, backend: str = "nccl", timeout_s: int = 120) -> None:
    if ws <= 1:
        return
    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def _device(backend: str):
    import torch

    return torch.device("cuda") if backend == "nccl" else torch.device("cpu")


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def reduce(ws: int, x: float, op: str = "max", backend: str = "nccl") -> float:
    """max or sum of x over the ranks (x itself on one rank)."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_device(backend))
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def shard(items: Sequence[T], rank: int, ws: int) -> list[T]:
    """The members this rank runs: every ws-th one from its rank on (all of
    them exactly once over the ranks)."""
    return [x for i, x in enumerate(items) if i % ws == rank]


def finish(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
