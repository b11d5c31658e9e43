"""Work split across ranks (one process per GPU).

Per-frame RMSD has no data exchange: frames are independent, so N ranks each
take a contiguous, balanced frame range, compute it on their own GPU and the
per-frame results are gathered at the end (a few bytes per frame).

The all-pairs matrix needs every frame on every rank, and splits the pairs:
the coordinate shards are all-gathered once into each rank's own memory
(240 MB for 20,000 frames x 1,000 atoms), each rank computes the tile rows of
the upper triangle that fall to it (wmd_pairwise_rmsd_part), and the parts
are summed.  No kernel reads another GPU's memory; the collectives are plain
torch.distributed calls (NCCL on GPUs, gloo on CPU).
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


def gather_frames(local, n_frames: int, group=None):
    """Every rank's frame shard (rank r holds frame_range(n_frames, r, world)),
    concatenated in rank order on every rank: one all_gather of equal-size
    padded blocks.  `local` is a tensor [f1 - f0, atoms, 3] on the rank's
    device (NCCL) or on the CPU (gloo); returns [n_frames, atoms, 3] there."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bounds = [frame_range(n_frames, r, world) for r in range(world)]
    f0, f1 = bounds[rank]
    if tuple(local.shape[:1]) != (f1 - f0,):
        raise RuntimeError(f"mismatch: rank {rank} holds {local.shape[0]} frames, its range has {f1 - f0}")
    width = max(b - a for a, b in bounds)
    block = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    block[: f1 - f0] = local
    blocks = [torch.empty_like(block) for _ in range(world)]
    dist.all_gather(blocks, block, group=group)
    return torch.cat([blk[: b - a] for (a, b), blk in zip(bounds, blocks)], dim=0)


def _cuda_part(frames, part: int, parts: int, metric: str, mode: str, sel=None):
    """This rank's part of the matrix on its own GPU (wmd_pairwise_rmsd_part),
    [F, F] float32 on the frames' device."""
    import torch

    from . import _native as N
    from .plans import _PAIR_MODES

    ctx = N.context(frames.device.index or 0)
    F, n_atoms = frames.shape[0], frames.shape[1]
    n_sel = n_atoms if sel is None else int(sel.shape[0])
    out = torch.empty((F, F), dtype=torch.float32, device=frames.device)
    m = {"rms": N.PAIR_RMS, "nofit": N.PAIR_NOFIT}[metric]
    stream = torch.cuda.current_stream(frames.device)
    ctx.check(ctx.lib.wmd_pairwise_rmsd_part(ctx.handle, frames.data_ptr(), F, n_atoms, frames.shape[2],
                                             None if sel is None else sel.data_ptr(), n_sel, m, _PAIR_MODES[mode],
                                             part, parts, out.data_ptr(), stream.cuda_stream))
    return out


def pairwise_sharded(local, n_frames: int, metric: str = "rms", mode: str = "i8x3", group=None,
                     dst: Optional[int] = None, compute_part: Optional[Callable] = None):
    """All-pairs RMSD matrix of a trajectory whose frames are split over the
    ranks (PairwiseRmsdPlan::finalize's i < j loop, plan.rs:593-674, split by
    tile rows).  Every rank passes its frame shard (frame_range order) and
    gets the [n_frames, n_frames] float32 matrix (every rank, or only rank
    `dst`; the others then get None).

    compute_part(frames, part, parts) -> [F, F] float32 computes one part; the
    default is this rank's GPU through wmd_pairwise_rmsd_part.  Each entry is
    written by exactly one part and is zero in all others, so the summed
    matrix equals the one-GPU matrix bit for bit."""
    import torch.distributed as dist

    if metric not in ("rms", "nofit"):
        raise RuntimeError("unsupported: the sharded all-pairs matrix takes metric 'rms' or 'nofit'")
    frames = gather_frames(local, n_frames, group)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if compute_part is None:
        mat = _cuda_part(frames, rank, world, metric, mode)
    else:
        mat = compute_part(frames, rank, world)
    if tuple(mat.shape) != (n_frames, n_frames):
        raise RuntimeError("mismatch: a part of the matrix has the wrong shape")
    del frames
    if dst is None:
        dist.all_reduce(mat, op=dist.ReduceOp.SUM, group=group)
        return mat
    dist.reduce(mat, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return mat if rank == dst else None


def pairwise_plan_sharded(plan, traj, system, group=None, device: Optional[str] = None):
    """PairwiseRmsdPlan.run split over the ranks: each rank takes its frame
    range of the selected atoms, and the matrix is assembled on every rank
    (numpy float32 [F, F]).  Metrics rms and nofit."""
    import torch
    import torch.distributed as dist

    from .plans import _check_inputs

    sel = _check_inputs(traj, system, plan.selection)
    n = traj.n_frames()
    f0, f1 = frame_range(n, dist.get_rank(group), dist.get_world_size(group))
    dev = torch.device(device) if device else torch.device("cuda", torch.cuda.current_device())
    local = torch.from_numpy(np.ascontiguousarray(traj.coords[f0:f1][:, sel], dtype=np.float32)).to(dev)
    return pairwise_sharded(local, n, metric=plan.metric, mode=plan.mode, group=group).cpu().numpy()
