"""Sharding of independent systems / requests over GPUs (one process per GPU).

Systems never interact, so the data path needs no collective: each rank relaxes its own
shard with its own copy of the grid.  The only collectives are a barrier and the
max-over-ranks of device times (the job's time is its slowest rank's).  This module holds
that host logic; it runs the same on NCCL (GPU tensors) and gloo (CPU tensors).
"""
from __future__ import annotations

import heapq

import numpy as np


def block_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) block of n items for a rank; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    q, r = divmod(int(n), world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def assign_by_cost(costs, world: int) -> list[np.ndarray]:
    """Longest-processing-time assignment of items with the given costs to `world` ranks:
    items in decreasing cost go to the least loaded rank (ties to the lower rank, equal costs in
    index order), so the result is deterministic.  Returns the sorted item indices per rank."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(int(i))
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def system_cost(natoms, rcut_pairs: float | None = None) -> np.ndarray:
    """Relative cost of relaxing systems of the given sizes: the NB partner loop is N^2 per step
    (every pair is visited; a cutoff only masks), bonded and grid work is linear."""
    n = np.asarray(natoms, dtype=np.float64)
    return n * n + 64.0 * n


def max_over_ranks(value: float) -> float:
    """Max of a float over all ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    """Sum of a float over all ranks of the default process group (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def grid_slabs(nx: int, world: int) -> tuple[int, list[tuple[int, int]]]:
    """Equal x-slabs for a sharded grid build: width ceil(nx / world) and each rank's [x0, x0 + width);
    the last slabs may reach past nx (their extra planes are computed and dropped), so the slabs
    concatenate in rank order under an all-gather of equal chunks."""
    if world <= 0:
        raise ValueError("world must be positive")
    w = -(-int(nx) // world)
    return w, [(r * w, r * w + w) for r in range(world)]


def gather_slabs(chunks, nx: int, ny: int, nz: int):
    """Host assembly of rank-ordered raw slabs (each 3 * width * ny * nz values) into the 3 * nx * ny * nz
    array of the whole grid: what the all-gather produces, trimmed to nx planes."""
    flat = np.concatenate([np.asarray(c).reshape(-1) for c in chunks])
    return flat[:3 * nx * ny * nz]


def build_grid_sharded(R, ions, ion_re, Lx, Ly, nx, ny, nz, p0, step, group=None, dtype=0, **params):
    """Substrate grid built across the ranks of a torch.distributed group (NCCL on GPUs): each rank
    evaluates the raw Morse and Ewald-2D values of its x-slab, one all-gather over NVLink replicates
    them, and every rank fits and installs the whole grid.  With one rank (or no process group) it
    is the single-GPU build split at the same point.  R: a RelaxMulti on this rank's GPU."""
    import torch
    import torch.distributed as dist
    ws = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if ws > 1 else 0
    w, slabs = grid_slabs(nx, ws)
    x0, _ = slabs[rank]
    local = torch.empty(3 * w * ny * nz, dtype=torch.float64, device="cuda")
    R.grid_raw_slab(ions, ion_re, Lx, Ly, nx, ny, nz, p0, step, x0, w, local.data_ptr(), **params)
    if ws > 1:
        full = torch.empty(ws * local.numel(), dtype=torch.float64, device="cuda")
        dist.all_gather_into_tensor(full, local, group=group)
    else:
        full = local
    torch.cuda.synchronize()
    R.grid_from_raw(full.data_ptr(), nx, ny, nz, p0, step, dtype=dtype)
    del local, full
