"""Query-sharded replicas, the multi-GPU form of the search.

The work shards by query with no exchange: every rank holds the whole index
and answers its own batch of the query stream.  The only collective is the
timing reduction (max over ranks), outside the data path.  Used by bench.py
under torchrun; tested with gloo ranks on the CPU.
"""
from __future__ import annotations

from . import datagen


def rank_queries(cfg: int, nq: int, rank: int):
    """Rank `rank`'s batch of the configuration's query stream: rank 0 gets
    the workload's own queries (seed 1235 + cfg), rank r the seed shifted by
    1000 r, all from the same distributions."""
    w = datagen.WORKLOADS[cfg]
    return datagen.make_queries(nq, w.zipf_s, w.n_labels, w.window, w.balanced_types, 1234 + cfg,
                                1235 + cfg + 1000 * rank)


def max_over_ranks(x: float, device: str = "cpu") -> float:
    """The largest value over all ranks (a step counts until its slowest rank
    ends).  device: "cuda" under NCCL, "cpu" under gloo."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, nq_per_rank: int, ms_per_step: float) -> float:
    """Whole-job queries/s: all ranks' queries over the slowest rank's step."""
    return world * nq_per_rank / (ms_per_step * 1e-3)
