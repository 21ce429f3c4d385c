"""Independent case replicas across ranks: one process per GPU.

UVLM cases never exchange data. The reference's only parallelism is `jax.vmap` over
stacked cases. Multi-GPU runs therefore shard cases over ranks, with no collective on
the data path. The only collectives are off it:
* the timing reduction (max over ranks);
* gathering the per-rank serving summaries.

Both run over NCCL on GPUs and over gloo on CPU.
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def rank_env() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Join the process group when the world has more than one rank. The short
    timeout makes ranks that wait for a rank that died end with an error."""
    import torch.distributed as dist

    rank, world, local = rank_env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def shard(items: list, rank: int, world: int) -> list:
    """This rank's cases: every world-th one, starting at the rank."""
    return list(items[rank::world])


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over all ranks (a device-timed duration)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(obj):
    """Every rank's object on rank 0 (a list in rank order); None elsewhere."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def merge_serving(parts: list[dict]) -> dict:
    """Whole-job serving summary from per-rank parts. Each part holds `case_steps`,
    `wall_s`, `gpu_busy_s`, `step_latency_ms` and `admit_latency_s` (lists) and
    `max_active`. Throughput is the case-steps of all ranks over the slowest rank's
    wall time. Latency percentiles are taken over every step of every rank."""
    steps = sum(p["case_steps"] for p in parts)
    wall = max(p["wall_s"] for p in parts)
    busy = max(p["gpu_busy_s"] for p in parts)
    lat = np.concatenate([np.asarray(p["step_latency_ms"], float) for p in parts]) if parts else np.zeros(0)
    adm = np.concatenate([np.asarray(p["admit_latency_s"], float) for p in parts]) if parts else np.zeros(0)
    pct = lambda a, q: float(np.percentile(a, q)) if a.size else None  # noqa: E731
    return {
        "case_steps": steps,
        "wall_s": wall,
        "steps_per_s": steps / wall if wall > 0 else None,
        "gpu_steps_per_s": steps / busy if busy > 0 else None,
        "p50_step_ms": pct(lat, 50),
        "p99_step_ms": pct(lat, 99),
        "mean_step_ms": float(lat.mean()) if lat.size else None,
        "p50_admit_s": pct(adm, 50),
        "p99_admit_s": pct(adm, 99),
        "max_active": max(p["max_active"] for p in parts),
        "ranks": len(parts),
    }
