"""Multi-GPU runs of the step: independent replicas, one process per GPU.

The ARW step's lateral boundary conditions belong to one domain, so N GPUs
run N independent integrations (ensemble members / seeds) with no data-path
collective.  The only communication is timing: a barrier around the timed
region and the maximum of the per-rank durations, from which the whole-job
rate is N * units / max_time.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> int:
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier() -> None:
    if world() > 1:
        dist.barrier()


def max_over_ranks(x: float) -> float:
    """The largest value of ``x`` over all ranks (``x`` itself on one rank)."""
    if world() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ms_max: float, nranks: int) -> float:
    """Whole-job throughput: every rank processed ``units_per_rank`` in at
    most ``ms_max`` milliseconds."""
    return nranks * units_per_rank / (ms_max / 1e3)
