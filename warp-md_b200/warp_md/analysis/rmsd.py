"""``pairwise_rmsd`` wrapper with the reference's arguments
(python/warp_md/analysis/rmsd.py:244-283): metric aliases ("srmsd" -> "rms"),
``mat_type`` "full" (N x N) or "half" (upper triangle, k=1, as float32)."""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from ..core import System, Trajectory
from ..plans import PairwiseRmsdPlan


def pairwise_rmsd(
    traj: Trajectory,
    system: System,
    mask: str = "",
    metric: str = "rms",
    mat_type: str = "full",
    pbc: str = "none",
    length_scale: float = 1.0,
    frame_indices: Optional[Sequence[int]] = None,
    chunk_frames: Optional[int] = None,
    device: str = "auto",
    mode: str = "fp64",
) -> np.ndarray:
    """Compute pairwise RMSD matrix (rms, nofit, dme, srmsd)."""
    aliases = {"srmsd": "rms"}
    metric = aliases.get(metric.lower(), metric.lower())
    mat_type, pbc = mat_type.lower(), pbc.lower()
    for name, value, allowed in (("metric", metric, ("rms", "nofit", "dme")),
                                 ("mat_type", mat_type, ("full", "half")),
                                 ("pbc", pbc, ("none", "orthorhombic"))):
        if value not in allowed:
            extra = " (or the alias 'srmsd')" if name == "metric" else ""
            raise ValueError(f"unknown {name} {value!r}: expected one of {', '.join(allowed)}{extra}")
    sel = system.select(mask if mask else "all")
    values = PairwiseRmsdPlan(sel, metric=metric, pbc=pbc, mode=mode).run(
        traj, system, chunk_frames=chunk_frames, device=device, frame_indices=frame_indices)
    # the reference scales the matrix, not the coordinates
    # (python/warp_md/analysis/rmsd.py:197)
    values = values * np.float32(length_scale)
    if mat_type == "full":
        return values
    if values.size == 0:
        return np.empty((0,), dtype=np.float32)
    tri = np.triu_indices(values.shape[0], k=1)
    return np.asarray(values[tri], dtype=np.float32)


__all__ = ["pairwise_rmsd"]
