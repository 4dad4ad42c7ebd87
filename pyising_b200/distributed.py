"""Ensembles across GPUs: one process per GPU, independent lattices sharded across ranks.

The sweep path shards naturally: lattices of an ensemble (temperature scans, Binder
ensembles, served jobs) are independent, so each rank runs its share with the batched kernels
of its own GPU and no collective touches the data path; only the finished (M, E) series (and
lattices, if kept) are gathered at the end over ``torch.distributed`` (NCCL on GPUs, gloo on
CPU).  Every lattice is bit-identical to running it alone, whichever rank runs it, because its
random numbers depend only on (site, sweep, colour, seed).
"""

from __future__ import annotations

from collections.abc import Callable, Sequence

import numpy as np


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-first greedy assignment of items with the given costs to ``world`` ranks.

    Deterministic (ties broken by index), so every rank computes the same plan without
    communicating.  Returns, per rank, the item indices in ascending order.
    """
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0.0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


def job_cost(job) -> float:
    """Work of a job in attempted spin updates (packed words cost less per update)."""
    return float(job.n_spins) * float(job.sweeps) * (0.25 if job.variant == "msc" else 1.0)


def run_local(jobs: Sequence, device: int = 0, memory_budget: float = 120e9) -> list:
    """Run jobs on this process's GPU in one batch; returns their results in order."""
    from .ensemble import Ensemble

    with Ensemble(device=device, memory_budget=memory_budget) as ens:
        ids = [ens.add(j) for j in jobs]
        ens.run()
        return [ens.result(i) for i in ids]


def run_sharded(jobs: Sequence, group=None, runner: Callable | None = None,
                gather_to: int | None = 0) -> list | None:
    """Run ``jobs`` sharded over the ranks of ``group`` (default: the default process group).

    Every rank must pass the same job list.  ``runner(sub_jobs) -> results`` runs one rank's
    share (default: :func:`run_local` on this rank's current CUDA device).  Results are gathered
    to rank ``gather_to`` (``None``: all ranks) and returned there in job order; other ranks
    return ``None``.
    """
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    plan = partition([job_cost(j) for j in jobs], world)
    mine = plan[rank]
    if runner is None:
        import torch

        dev = torch.cuda.current_device() if torch.cuda.is_available() else 0
        results = run_local([jobs[i] for i in mine], device=dev)
    else:
        results = runner([jobs[i] for i in mine])
    payload = [(i, _to_host(r)) for i, r in zip(mine, results, strict=True)]
    if world == 1:
        gathered = [payload]
    elif gather_to is None:
        gathered = [None] * world
        dist.all_gather_object(gathered, payload, group=group)
    else:
        gathered = [None] * world if rank == gather_to else None
        dist.gather_object(payload, gathered, dst=gather_to, group=group)
        if rank != gather_to:
            return None
    out: list = [None] * len(jobs)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out


def _to_host(result):
    """Results travel as plain NumPy (series, lattice) pairs."""
    series = np.asarray(result.series)
    lattice = None if result.lattice is None else np.asarray(result.lattice)
    return type(result)(series, lattice) if hasattr(result, "series") else result
