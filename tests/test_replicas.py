"""Multi-rank plumbing on CPU: two gloo ranks (spawned processes) shard cases, reduce
the timing to its maximum and merge serving summaries on rank 0 -- the collectives the
GPU runs make over NCCL, none of them on the data path."""
from __future__ import annotations

import json
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch.distributed as dist

    from flapjax_b200 import replicas

    r, w, _ = replicas.init("gloo", timeout_s=60)
    cases = list(range(10))
    mine = replicas.shard(cases, r, w)
    t = replicas.max_over_ranks(1.5 + r)  # the slowest rank's time wins
    part = {"case_steps": 10 * len(mine), "wall_s": 2.0 + r, "gpu_busy_s": 1.0 + r,
            "step_latency_ms": [1.0 + r] * (10 * len(mine)), "admit_latency_s": [0.1 * (r + 1)] * len(mine),
            "max_active": 3 + r}
    parts = replicas.gather_to_root(part)
    merged = replicas.merge_serving(parts) if parts is not None else None
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"mine": mine, "t": t, "merged": merged}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_reduce_and_merge(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert r0["mine"] == [0, 2, 4, 6, 8] and r1["mine"] == [1, 3, 5, 7, 9]
    assert r0["t"] == r1["t"] == 2.5
    m = r0["merged"]
    assert r1["merged"] is None
    assert m["case_steps"] == 100 and m["wall_s"] == 3.0 and m["ranks"] == 2
    assert m["steps_per_s"] == pytest.approx(100 / 3.0)
    assert m["p50_step_ms"] == pytest.approx(1.5) and m["max_active"] == 4


def test_single_process_needs_no_group():
    from flapjax_b200 import replicas

    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
    assert replicas.max_over_ranks(4.0) == 4.0
    assert replicas.gather_to_root({"a": 1}) == [{"a": 1}]
