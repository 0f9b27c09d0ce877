"""Multi-GPU host logic: one process per GPU, GRGs (genomic regions) sharded across ranks.

A single GRG traversal is level-synchronous and does not shard without a per-level exchange,
so the hot path stays on one GPU.  What shards is the set of GRGs: the reference already loads
each artifact independently per device (``pygrgl_spmv/adaptor.py:983-1051``) and callers sum
the per-region ``down`` results (``scripts/bolt_lmm_inf/core.py:1282-1301``); ``down`` over a
genome split into regions equals the sum of the regions' ``down`` outputs
(``pygrgl_spmv/tests/endtoend/test_matmul.py:255-299``).  ``up`` outputs are disjoint mutation
ranges and need no collective.

* ``assign_regions``: balanced, deterministic region -> rank assignment (largest first onto
  the least-loaded rank, by edge count).
* ``sum_region_down``: the one real exchange, an all-reduce SUM of ``[samples, k]`` (NCCL over
  NVLink/NVSwitch on GPUs, gloo in the CPU tests).
* ``reduce_job_time``: whole-job throughput bookkeeping (max time over ranks, summed work).
"""

from __future__ import annotations

from collections.abc import Sequence


def assign_regions(region_edges: Sequence[int], world_size: int) -> list[list[int]]:
    """Indices of the regions each rank owns; every region is owned by exactly one rank."""
    world_size = int(world_size)
    if world_size < 1:
        raise ValueError(f"world_size must be >= 1, got {world_size}")
    load = [0] * world_size
    owned: list[list[int]] = [[] for _ in range(world_size)]
    order = sorted(range(len(region_edges)), key=lambda i: (-int(region_edges[i]), i))
    for region in order:
        rank = min(range(world_size), key=lambda r: (load[r], r))
        owned[rank].append(region)
        load[rank] += int(region_edges[region])
    return [sorted(regions) for regions in owned]


def sum_region_down(partial, group=None):
    """All-reduce SUM, in place, of this rank's summed region ``down`` outputs."""
    import torch.distributed as dist

    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


def reduce_job_time(elapsed_ms: float, work: float, device=None, group=None) -> tuple[float, float]:
    """(max elapsed ms over ranks, total work over ranks)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(elapsed_ms), float(work)
    t = torch.tensor([float(elapsed_ms)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(w, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), float(w.item())


__all__ = ["assign_regions", "reduce_job_time", "sum_region_down"]
