"""Frame sharding across ranks (one process per GPU).

The RMSD path has no data exchange: frames are independent, so N ranks each
take a contiguous, balanced frame range, compute it on their own GPU and the
per-frame results are gathered at the end (a few bytes per frame).  Nothing
but that gather -- and the max-over-ranks timing in the benchmark -- crosses
ranks.  ``torch.distributed`` carries the gather: NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np


def frame_range(n_frames: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced [f0, f1) of rank `rank` out of `world`."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("invalid rank/world")
    return n_frames * rank // world, n_frames * (rank + 1) // world


def gather_series(local: np.ndarray, n_frames: int, group=None) -> np.ndarray:
    """Concatenates every rank's slice (in rank order) on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    bounds = [frame_range(n_frames, r, world) for r in range(world)]
    width = max(b - a for a, b in bounds)
    buf = torch.zeros(width, dtype=torch.float64, device=dev)
    buf[: local.shape[0]] = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty(n_frames, np.float64)
    for (a, b), p in zip(bounds, parts):
        out[a:b] = p[: b - a].cpu().numpy()
    return out


def run_sharded(compute: Callable[[int, int], np.ndarray], n_frames: int, group=None) -> np.ndarray:
    """Runs compute(f0, f1) on this rank's frames and gathers all ranks'."""
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    f0, f1 = frame_range(n_frames, rank, world)
    local = np.asarray(compute(f0, f1), dtype=np.float64)
    if local.shape != (f1 - f0,):
        raise RuntimeError("mismatch: shard result has the wrong length")
    return gather_series(local, n_frames, group)


def rmsd_plan_sharded(plan, traj, system, group=None, device: Optional[str] = None, **kw) -> np.ndarray:
    """RmsdPlan.run over this rank's frame range on its own GPU, gathered.
    Frame0 mode uses frame 0 of the whole trajectory on every rank."""
    import torch

    dev = device or f"cuda:{torch.cuda.current_device()}"
    n = traj.n_frames()
    if plan.reference_mode == "frame0":
        from .core import System
        from .plans import RmsdPlan

        ref_system = System(system.names, system.resnames, system.resids, system.masses, system.elements,
                            system.chains, traj.coords[0])
        plan = RmsdPlan(plan.selection, reference="topology", align=plan.align)
        system = ref_system

    def compute(f0: int, f1: int) -> np.ndarray:
        return plan.run(traj, system, device=dev, frame_indices=list(range(f0, f1)), dtype=np.float64, **kw)

    return run_sharded(compute, n, group)
