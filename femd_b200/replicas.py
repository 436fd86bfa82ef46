"""The multi-GPU form of this path: independent replicas, one process per GPU, no collective on
the data path.  Every rank serves its own copy of the workload; the only collectives are a
barrier around the timed region and the max over ranks of the measured time.  A short
process-group timeout turns a rank that never arrives into an error on the others instead of a
hang."""
from __future__ import annotations

import datetime
import os


def init(backend: str, timeout_s: float = 120.0):
    """torch.distributed from the launcher's environment (RANK, WORLD_SIZE, MASTER_*); returns
    the dist module, or None when WORLD_SIZE is 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    import torch.distributed as D
    D.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return D


def max_over_ranks(t: float, dist, device: str = "cuda") -> float:
    """The slowest rank's time (every rank takes part; gloo on CPU tensors, NCCL on CUDA)."""
    if dist is None:
        return t
    import torch
    v = torch.tensor([t], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


def whole_job_value(units_per_rank: float, world: int, t_max: float) -> float:
    """Throughput of the whole job: every rank's units over the slowest rank's time (weak
    scaling: each rank does the same work)."""
    return world * units_per_rank / t_max


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
