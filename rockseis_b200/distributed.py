"""Shots across GPUs: cost-balanced shot partition and one reduction of the stacked
gradient at the end.

The reference spreads shots over MPI workers from a master queue
(lib/parallel.cpp, Inversion*::runGrad lib/inversion.cpp:231-602) and stacks the
per-shot gradients through files (`stackImage`).  Shots are independent, so here
each rank (one process per GPU, torch.distributed) takes a fixed share of the shots,
computes their gradients in one batched GPU run, sums them in FP64 on the host, and
one all-reduce over the ranks (NCCL on GPUs, gloo on CPUs) stacks the result and the
misfit.  There is no exchange inside the time loop.
"""
from __future__ import annotations

import heapq

import numpy as np


def shot_cost(model, nt: int) -> float:
    """Work of one shot: padded points of its window x time steps."""
    return float(model.getNx_pml()) * float(model.getNz_pml()) * float(model.getNy_pml()) * float(nt)


def partition_shots(costs, world: int) -> list[list[int]]:
    """Shot indices per rank, balancing the summed cost: longest-processing-time
    first (largest shot to the least loaded rank, ties to the lower rank), each
    rank's list in ascending shot order.  Deterministic, so every rank computes the
    same partition without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def _allreduce_sum(vec: np.ndarray, group=None) -> np.ndarray:
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(vec, np.float64))
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def _default_runner(jobs):
    from .rockseis import fwi_gradient_batch
    fwi_gradient_batch(jobs)


def fwi_gradient_sharded(jobs, rank: int, world: int, group=None, runner=None):
    """Stacked FWI gradient of all `jobs` (FwiAcoustic2D-like objects on one model
    grid, every rank holding the same list) computed by `world` ranks.

    Rank `rank` runs its share (partition_shots over shot_cost) through `runner`
    (default: one batched rsgpu_fwi_gradient call), which fills each job's vpgrad /
    rhograd images and misfit.  Returns (vpgrad, rhograd, misfit) summed over all
    shots in FP64, identical on every rank."""
    if not jobs:
        raise ValueError("no shots")
    shape = jobs[0].vpgrad.getImagedata().shape
    for j in jobs:
        if j.vpgrad.getImagedata().shape != shape or j.rhograd.getImagedata().shape != shape:
            raise ValueError("sharded stacking needs every shot's gradient on the same grid")
    mine = partition_shots([shot_cost(j.model, j.source.nt) for j in jobs], world)[rank]
    local = [jobs[i] for i in mine]
    if local:
        (runner or _default_runner)(local)
    n = int(np.prod(shape))
    vec = np.zeros(2 * n + 1, np.float64)
    for j in local:
        vec[:n] += j.vpgrad.getImagedata().reshape(-1)
        vec[n:2 * n] += j.rhograd.getImagedata().reshape(-1)
        vec[2 * n] += float(j.misfit)
    if world > 1:
        vec = _allreduce_sum(vec, group)
    return vec[:n].reshape(shape), vec[n:2 * n].reshape(shape), float(vec[2 * n])
