"""Instance sharding of a decomposition job across GPUs, one process per GPU.

Epochs (and, for SMP, channels) share nothing: each has its own residual and
maps, and the dictionary depends only on (fs, N, energyError).  A job is
therefore split across ranks with no collective on the data path: every rank
decomposes its share on its own GPU and the atoms are gathered on rank 0.

    parts = partition(costs, world)            # greedy longest-first
    results = decompose_sharded(variant, epochs, fs, ...)   # rank 0: all, others: None
"""
from __future__ import annotations

import heapq
import math


def epoch_cost(shape, fs, energy_error, iterations, variant, scale_min=0.0, scale_max=math.inf,
               freq_max=math.inf) -> float:
    """Relative work of one epoch: dictionary size x MP loops x (initial pass +
    about half a pass per iteration, the refresh region of a mid-scale atom)."""
    import ctypes

    from empi_b200 import Dictionary, _check, load_library

    n, c = shape
    d = Dictionary(float(energy_error), float(scale_min), float(scale_max), float(freq_max))
    count = ctypes.c_uint64()
    _check(load_library().empi_dictionary_size(ctypes.byref(d), float(fs), int(n), ctypes.byref(count), None))
    loops = 1 if variant == "mmp2" else c
    return float(count.value) * loops * (1.0 + 0.5 * iterations)


def partition(costs, world):
    """Greedy longest-processing-time split: indices per rank, each list in
    ascending index order; every index appears exactly once."""
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def decompose_sharded(variant, epochs, fs, energy_error, iterations, energy_percent=100.0, scale_min=0.0,
                      scale_max=math.inf, freq_max=math.inf, group=None, decompose_fn=None, costs=None,
                      engine=None):
    """Decomposes `epochs` (list of (N, C) float32 arrays, identical on every
    rank) across the ranks of `group`; returns the per-epoch results in order
    on rank 0 and None elsewhere.  decompose_fn(variant, epochs, fs, ...)
    defaults to empi_b200.decompose_epochs on this rank's GPU: `engine`, or
    an engine on device LOCAL_RANK."""
    import os

    import torch.distributed as dist

    if decompose_fn is None:
        import empi_b200

        eng = engine or empi_b200.Engine(device=int(os.environ.get("LOCAL_RANK", "0")))

        def decompose_fn(*args):
            return empi_b200.decompose_epochs(*args, engine=eng)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if costs is None:
        costs = [epoch_cost(e.shape, fs, energy_error, iterations, variant, scale_min, scale_max, freq_max)
                 for e in epochs]
    parts = partition(costs, world)
    mine = parts[rank]
    local = decompose_fn(variant, [epochs[i] for i in mine], fs, energy_error, iterations, energy_percent,
                         scale_min, scale_max, freq_max) if mine else []
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, local)), gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(epochs)
    for chunk in gathered:
        for i, res in chunk:
            out[i] = res
    return out
