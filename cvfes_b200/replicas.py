"""Replica ensembles across ranks (one process per GPU).

Samples never interact (each sample's step reads only its own state, as the reference's
per-sample loop does, ``physicsSolverSDampGPUs.cl:264``), so more GPUs run more
independent ensembles: rank r advances its own ensemble, drawn from GMRF seeds offset by
``1000 * r``, with no collective on the data path.  The only collectives are on the
host side of a measurement: the slowest rank's time (``max_over_ranks``) and totals
(``sum_over_ranks``).  They run on whatever process group is initialised (NCCL between
GPUs, gloo on the CPU) and are the identity without one.
"""
from __future__ import annotations

import dataclasses

import torch
import torch.distributed as dist

SEED_STRIDE = 1000


def rank_case(case, rank: int):
    """The workload of rank ``rank``: the same mesh and sizes, its own material seeds."""
    return dataclasses.replace(case, seed_E=case.seed_E + SEED_STRIDE * rank,
                               seed_h=case.seed_h + SEED_STRIDE * rank)


def _reduce(value: float, op, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Largest value over all ranks (a timed region is as long as its slowest rank)."""
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, device=None) -> float:
    """Sum over all ranks (work done by the whole job)."""
    return _reduce(value, dist.ReduceOp.SUM, device)
