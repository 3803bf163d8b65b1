"""Multi-GPU runs as independent replicas: one process per GPU, each rendering
its own frame-seed sequence of the same workload. Pixels, paths and frames
are independent, so the data path has no collective; torch.distributed is
used only for the start/stop barrier and the max-over-ranks step time.

The whole-job throughput is all ranks' paths divided by the slowest rank's
device time (weak scaling: the per-rank work is fixed as ranks are added).
"""
from __future__ import annotations

import datetime
import os

# Frame seeds of rank r start at r * SEED_STRIDE; a run must use fewer than
# SEED_STRIDE consecutive seeds per rank so that no two ranks share a path.
SEED_STRIDE = 1_000_003


def env_ranks():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 300.0):
    """Join the process group when WORLD_SIZE > 1 (rendezvous from MASTER_ADDR /
    MASTER_PORT); returns (world_size, rank, local_rank)."""
    ws, rank, local = env_ranks()
    if ws > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return ws, rank, local


def seed_base(rank: int) -> int:
    return rank * SEED_STRIDE


def check_seed_budget(seeds_per_rank: int) -> None:
    if seeds_per_rank >= SEED_STRIDE:
        raise ValueError(f"{seeds_per_rank} frame seeds per rank overlap the next rank's (stride {SEED_STRIDE})")


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws: int, x: float, device: str = "cuda") -> float:
    """The largest x over all ranks (every rank gets it)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, ws: int, ms_max: float) -> float:
    """All ranks' units per second of the slowest rank's time, in millions."""
    return units_per_rank * ws / (ms_max * 1e-3) / 1e6


def finish(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
