"""``rotation_matrix`` with the reference's arguments
(python/warp_md/analysis/rotation.py:190-279): per-frame rotations (frames,
3, 3) float32 that superpose each frame's ``mask`` atoms onto the reference;
frames outside ``frame_indices`` keep the identity (and RMSD 0)."""
from __future__ import annotations

from typing import Optional, Sequence, Union

import numpy as np

from ..plans import frame_subset, superpose_arrays
from .align import _indices, _masses, reference_coords
from .trajectory import read_all_frames

RefLike = Union[int, str]


def rotation_matrix(traj, system, mask: str = "", ref: RefLike = 0, mass: bool = False,
                    frame_indices: Optional[Sequence[int]] = None, chunk_frames: Optional[int] = None,
                    with_rmsd: bool = False, device: str = "auto"):
    """Compute rotation matrices to align frames to reference."""
    coords, _box, _time = read_all_frames(traj, chunk_frames)
    if coords is None:
        raise ValueError("trajectory has no frames")
    n = coords.shape[0]
    mats = np.broadcast_to(np.eye(3, dtype=np.float32), (n, 3, 3)).copy()
    rmsd = np.zeros(n, dtype=np.float32) if with_rmsd else None
    if n:
        idx = _indices(system, mask)
        ref_xyz = np.asarray(reference_coords(coords, system, ref), dtype=np.float32)[idx]
        sub = frame_subset(n, frame_indices)
        rows = np.arange(n) if sub is None else sub
        if rows.size:
            xf, _ = superpose_arrays(coords[rows], idx, ref_xyz, _masses(system, idx, mass), False, False, device)
            mats[rows] = xf[:, :9].reshape(-1, 3, 3)
            if with_rmsd:
                from ..plans import RmsdPlan
                from ..core import Selection, System, Trajectory

                sys2 = System([""] * coords.shape[1], None, None, None, None, None, None)
                sys2.positions0 = np.zeros((coords.shape[1], 3), np.float32)
                sys2.positions0[idx] = ref_xyz
                vals = RmsdPlan(Selection(idx), reference="topology").run(
                    Trajectory(np.ascontiguousarray(coords[rows])), sys2, device=device)
                rmsd[rows] = vals
    return (mats, rmsd) if with_rmsd else mats


__all__ = ["rotation_matrix"]
