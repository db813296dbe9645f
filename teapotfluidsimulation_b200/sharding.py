"""Multi-GPU sharding of the work that shards: ensembles of pours and batches of Poisson snapshots.

A single pour does not shard (its liquid system is a few thousand to ~100k unknowns, coupled every
substep), so N GPUs run N independent replicas of it. Ensembles and snapshot batches are sets of
independent units: each rank runs its own share with no collective on the data path, and the only
exchange is a final gather of about a hundred bytes of stats per unit. The grids are uneven, so the
units are partitioned by estimated cost, not by index.

Cost model (relative; only the ratios between units matter):
  - a pour: (cells + parcels) x estimated substeps. Every stage of a substep is a pass over the cells
    or over the parcels, and the substep count is the duration over the CFL step bound with the free-
    fall speed of the fill height (solver3d.ts:268-278), capped by the maximum substep;
  - a snapshot: its unknowns (multigrid PCG iterations are nearly flat across these masks).
"""
from __future__ import annotations

import math

import numpy as np

from . import abi


def partition_by_cost(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of units to `world` ranks: units in decreasing cost
    (ties by index) each go to the rank with the smallest load so far (ties by rank). Deterministic, so
    every rank computes the same partition without communicating. Returns each rank's unit indices in
    increasing order. The largest load is at most 4/3 of the optimum (Graham's bound)."""
    costs = [float(c) for c in costs]
    if world < 1:
        raise ValueError("world must be >= 1")
    if any(not math.isfinite(c) or c < 0 for c in costs):
        raise ValueError("costs must be finite and non-negative")
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def estimated_substeps(cfg: abi.Config, fill_height: float) -> float:
    """Substeps of a pour of `cfg.duration` seconds: CFL bound with the free-fall speed of the fill
    height plus the sqrt(5 h g) term of stableDt (solver3d.ts:268-278), capped by max_substep."""
    speed = math.sqrt(2 * cfg.gravity * max(fill_height, 0.0)) + math.sqrt(5 * cfg.h * cfg.gravity)
    dt = min(cfg.max_substep, cfg.cfl * cfg.h / speed)
    return cfg.duration / dt


def pour_costs(cfgs) -> list[float]:
    """Estimated cost of each pour (host construction only, no device: pl_plan)."""
    from .engine import plan

    out = []
    for cfg in cfgs:
        s = plan(cfg)["sizes"]
        out.append((s.nx * s.ny * s.nz + s.n) * estimated_substeps(cfg, s.fill_height))
    return out


def snapshot_costs(n: int, first: int, count: int) -> list[float]:
    """Unknowns of snapshots first .. first+count-1 of the synthetic Poisson batch (masks only)."""
    import ctypes as C

    from .engine import _check, lib

    cell = np.zeros((count, n * n * n), np.uint8)
    _check(lib().pl_poisson_generate(n, first, count, cell.ctypes.data_as(C.POINTER(C.c_uint8)), None, 0))
    return [float(v) for v in ((cell & 3) == abi.FLUID).sum(axis=1)]


def contiguous_runs(indices) -> list[tuple[int, int]]:
    """(first, count) runs of sorted indices, for generators that take contiguous ranges."""
    runs: list[tuple[int, int]] = []
    for i in sorted(indices):
        if runs and runs[-1][0] + runs[-1][1] == i:
            runs[-1] = (runs[-1][0], runs[-1][1] + 1)
        else:
            runs.append((i, 1))
    return runs


def gather_stats(local: dict, world: int) -> dict:
    """Every rank's {unit index: stats} merged on every rank (one all_gather of Python objects; a
    single process returns its own). Raises if two ranks report the same unit."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    got = [None] * world
    dist.all_gather_object(got, local)
    merged: dict = {}
    for part in got:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"unit {k} reported by two ranks")
            merged[k] = v
    return merged
