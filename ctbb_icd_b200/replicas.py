"""Independent reconstructions: the batched-scan workload and its split
across GPUs.

A reconstruction does not shard (every voxel update reads and writes the one
error sinogram of its scan), so several GPUs run independent scans: one
process per GPU, scans assigned up front by estimated cost, no data-path
collective. The only collective is the max-over-ranks of the timed region.
"""
from __future__ import annotations

import math
import random

from . import workloads as W


def batch_specs(n: int = 32, seed: int = 0) -> list[dict]:
    """The uneven batch: n seeded helical scans (parameter-file dicts plus
    phantom), matrix size from {128,256,384,512}^2, rows from {8,16,32,64},
    pitch uniform in 0.5..1.5, with or without the in-plane flying focal
    spot, 8..64 slices; quadratic penalty, 20 iterations, random-ellipsoid
    phantoms."""
    rng = random.Random(seed)
    out = []
    for i in range(n):
        nx = rng.choice([128, 256, 384, 512])
        rows = rng.choice([8, 16, 32, 64])
        pitch = rng.uniform(0.5, 1.5)
        ffs = rng.random() < 0.5
        nz = rng.randint(8, 64)
        row_iso = 0.06 if rows >= 32 else 0.12
        views_wo = 1152
        vz = row_iso  # slice thickness = detector row width at isocentre
        # Enough turns for the slab plus the system-matrix window on both sides.
        feed = pitch * rows * row_iso
        turns = int(math.ceil((nz * vz + 2.0 * rows * row_iso * 1.3) / feed)) + 2
        prm = {**W._BASE,
               **W._scanner(736, 366.25, W.FAN_INC, rows, row_iso, views_wo, ffs, pitch, turns),
               **W._recon(nx, 30.0, vz, nz, -1.0, "quadratic", 0.1, 0.005, 20)}
        z_first = (turns * views_wo * (2 if ffs else 1) / (views_wo * (2 if ffs else 1))) * feed / 10.0
        # Centre the slab in the scanned range (the window of setup.cpp:359-371).
        span = turns * feed
        z_start = z_first - 0.5 * span + 0.5 * nz * vz
        prm.update(z_start=z_start, z_end=z_start - (nz + 0.5) * vz)
        out.append(dict(name=f"scan{i:02d}", prm=prm,
                        phantom=dict(n_ellipsoids=40, seed=seed * 1000 + i, i0_lo=5e4, i0_hi=2e5)))
    return out


def scan_cost(spec: dict) -> float:
    """Relative cost of one iteration: voxels x matrix entries per voxel
    (entries grow with the rows a slice spans and the views in its window)."""
    p = spec["prm"]
    voxels = p["nx"] * p["ny"] * round(abs(p["z_end"] - p["z_start"]) / p["slice_thickness"])
    views = p["num_views_per_turn_without_ffs"] * (2 if p["Phiffs"] else 1)
    return float(voxels) * views * (1.0 / p["nx"]) * max(1.0, p["slice_thickness"] / p["CollSlicewidth"])


def assign(costs: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of scans to ranks
    (deterministic: ties broken by index)."""
    loads = [0.0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        r = min(range(world), key=lambda k: (loads[k], k))
        plan[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in plan]


def my_scans(costs: list[float], world: int, rank: int) -> list[int]:
    return assign(costs, world)[rank]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (the timed region's duration) over ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
