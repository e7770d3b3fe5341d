"""Independent replicas across ranks: one process per GPU, no data-path collective.

The step does not shard without a per-step exchange (the global min-tau and the face-crossing
diffusion counts), so multi-GPU work is replicas: rank r advances its own copy of the model on its
own random stream, keyed by (seed, replica = r) in the Philox key, and the ranks meet only to
combine their measurements: device time is the maximum over ranks (the job ends when the slowest
rank ends), events and simulated time are summed.  The functions take a torch.distributed module
(or None for a single process) and run on any backend: NCCL with CUDA tensors on a GPU box, gloo
with CPU tensors in the tests.
"""
from __future__ import annotations

import os
from typing import Dict, Optional


def rank_env() -> tuple:
    """(world_size, rank, local_rank) from the torchrun environment, (1, 0, 0) without it."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_options(rank: int, seed: int = 1000) -> Dict[str, int]:
    """Stream of rank `rank`: the common seed with the rank as replica id, so every rank draws from
    a different Philox key and any single rank can be replayed alone (Simulation(..., **opts))."""
    return {"seed": int(seed), "replica": int(rank)}


def combine(dist, device, *, max_keys: Dict[str, float], sum_keys: Dict[str, float]) -> Dict[str, float]:
    """Whole-job figures: every entry of max_keys reduced with MAX over ranks, every entry of
    sum_keys with SUM.  All ranks must call it with the same keys in the same order (one
    collective each for the two groups).  dist None: returns the inputs."""
    out = dict(max_keys)
    out.update(sum_keys)
    if dist is None:
        return out
    import torch
    for keys, op in ((list(max_keys), dist.ReduceOp.MAX), (list(sum_keys), dist.ReduceOp.SUM)):
        if not keys:
            continue
        src = max_keys if op == dist.ReduceOp.MAX else sum_keys
        t = torch.tensor([float(src[k]) for k in keys], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        for k, v in zip(keys, t.tolist()):
            out[k] = v
    return out


def init(backend: str, local_rank: int, timeout_s: float = 120.0):
    """Join the process group of a torchrun launch (short timeout, so that ranks waiting for a rank
    that died end with an error instead of waiting for good).  Returns the torch.distributed module,
    or None for a single process."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def finish(dist) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def rank_device(dist, local_rank: int) -> Optional[str]:
    """Device of the tensors combine() reduces: the rank's GPU under NCCL, the CPU under gloo."""
    if dist is None:
        return None
    return f"cuda:{local_rank}" if dist.get_backend() == "nccl" else "cpu"
