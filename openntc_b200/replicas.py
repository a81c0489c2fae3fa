"""Replica parallelism across GPUs: one process per GPU, independent materials per process.

One material does not shard (its latents are dense per level and its decoder is shared by
every texel), but a set of materials does: each rank trains (or decodes) its own share and
the ranks only exchange host-side scalars at the end -- the largest per-rank time and the
per-material results.  Nothing moves through the data path between GPUs.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class MaterialSpec:
    """One material of a batch job: its texture size, channel count, profile and schedule."""
    name: str
    dim: int
    channels: int
    profile: int
    steps: int
    grids_per_batch: int = 1

    def cost(self) -> float:
        """Texels trained over the schedule: steps x tiles x (min(mip, 256))^2 at the top mip,
        the quantity the training time scales with (upstream trains min(mip, 256)^2 texels
        per tile, libopenntc.cpp:564-585)."""
        t = min(self.dim, 256)
        return float(self.steps) * self.grids_per_batch * t * t


def partition(costs: list[float], world: int) -> list[list[int]]:
    """Deterministic longest-processing-time split of items over `world` ranks: items in
    decreasing cost (ties by index) each go to the least-loaded rank (ties by rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for items in out:
        items.sort()
    return out


def env_rank() -> tuple[int, int, int]:
    """(world, rank, local_rank) from the launcher's environment (torchrun / torch.distributed.run)."""
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ReplicaGroup:
    """The host-side exchange between replicas.  With world == 1 every call is local."""

    def __init__(self, world: int, rank: int, backend: str | None = None, timeout_s: float = 300.0):
        self.world, self.rank = world, rank
        self.dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, value: float) -> float:
        """Largest value over the ranks (every rank gets it)."""
        if not self.dist:
            return value
        vals = [None] * self.world
        self.dist.all_gather_object(vals, float(value))
        return max(vals)

    def gather(self, obj):
        """Every rank's object, in rank order (every rank gets the list)."""
        if not self.dist:
            return [obj]
        vals = [None] * self.world
        self.dist.all_gather_object(vals, obj)
        return vals

    def close(self):
        if self.dist and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None


def run_share(specs: list[MaterialSpec], group: ReplicaGroup, work) -> dict[str, object]:
    """Runs `work(spec)` for this rank's share of `specs` (cost-model partition) and returns
    every rank's results by material name, on every rank."""
    share = partition([s.cost() for s in specs], group.world)[group.rank]
    local = {specs[i].name: work(specs[i]) for i in share}
    merged: dict[str, object] = {}
    for part in group.gather(local):
        merged.update(part)
    return merged
