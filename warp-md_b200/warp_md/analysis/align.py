"""``align`` / ``superpose`` with the reference's arguments
(python/warp_md/analysis/align.py:167-267): frames superposed onto a
reference frame (an integer index) or the topology coordinates, over the
``mask`` atoms (optionally mass-weighted); every atom of a frame moves by its
frame's transform.  Returns an ArrayTrajectory."""
from __future__ import annotations

from typing import Optional, Sequence, Union

import numpy as np

from ..plans import frame_subset, superpose_arrays
from .trajectory import ArrayTrajectory, read_all_frames

RefLike = Union[int, str]


def _indices(system, mask: str) -> np.ndarray:
    sel = system.select(mask if mask else "all")
    return np.asarray(list(sel.indices), dtype=np.int64)


def _masses(system, idx: np.ndarray, mass: bool) -> Optional[np.ndarray]:
    if not mass:
        return None
    if hasattr(system, "masses"):
        masses = np.asarray(system.masses, dtype=np.float32)
    else:
        masses = np.asarray(system.atom_table().get("mass", []), dtype=np.float32)
    if masses.size == 0:
        return None
    return np.ascontiguousarray(masses[idx], dtype=np.float32)


def reference_coords(coords: np.ndarray, system, ref: RefLike) -> np.ndarray:
    """resolve_reference_coords (python/warp_md/analysis/_runtime.py:306-335):
    an integer frame index, "topology" (positions0, else frame 0) or
    "frame0"."""
    if isinstance(ref, (int, np.integer)):
        i = int(ref)
        if i < 0 or i >= coords.shape[0]:
            raise ValueError("ref index out of range")
        return coords[i]
    if not isinstance(ref, str):
        raise ValueError("ref must be an integer frame index or a supported string")
    key = ref.strip().lower()
    if key in ("topology", "top", "topo"):
        p0 = getattr(system, "positions0", None)
        if callable(p0):
            p0 = p0()
        if p0 is not None:
            return np.asarray(p0, dtype=np.float32)
        return reference_coords(coords, system, 0)
    if key in ("frame0", "first", "0"):
        return reference_coords(coords, system, 0)
    raise ValueError("unsupported ref value")


def _transforms(coords, system, mask, ref, ref_mask, mass, device):
    idx = _indices(system, mask)
    ref_idx = _indices(system, ref_mask)
    if idx.size != ref_idx.size:
        raise ValueError("mask and ref_mask selections must have same size")
    ref_xyz = np.asarray(reference_coords(coords, system, ref), dtype=np.float32)[ref_idx]
    return idx, ref_xyz, _masses(system, idx, mass)


def align(traj, system, mask: str = "", ref: RefLike = 0, ref_mask: Optional[str] = None, mass: bool = False,
          chunk_frames: Optional[int] = None, return_transforms: bool = False, device: str = "auto"):
    """Align trajectory frames to a reference via Kabsch."""
    ref_mask = mask if ref_mask is None else ref_mask
    coords, box, time = read_all_frames(traj, chunk_frames)
    if coords is None:
        raise ValueError("trajectory has no frames")
    if coords.size == 0:
        out = ArrayTrajectory(coords, box=box, time_ps=time)
        return (out, np.empty((0, 12), dtype=np.float32)) if return_transforms else out
    idx, ref_xyz, w = _transforms(coords, system, mask, ref, ref_mask, mass, device)
    xf, moved = superpose_arrays(coords, idx, ref_xyz, w, False, True, device)
    out = ArrayTrajectory(moved, box=box, time_ps=time)
    return (out, xf) if return_transforms else out


def superpose(traj, system, mask: str = "", ref: RefLike = 0, ref_mask: Optional[str] = None, mass: bool = False,
              frame_indices: Optional[Sequence[int]] = None, chunk_frames: Optional[int] = None,
              device: str = "auto"):
    """Superpose trajectory frames to a reference (returns aligned coords);
    with ``frame_indices`` only those frames move, the others are returned
    unchanged (align.py:225-267)."""
    ref_mask = mask if (ref_mask is None or ref_mask == "") else ref_mask
    coords, box, time = read_all_frames(traj, chunk_frames)
    if coords is None:
        raise ValueError("trajectory has no frames")
    if coords.size == 0:
        return ArrayTrajectory(coords, box=box, time_ps=time)
    idx, ref_xyz, w = _transforms(coords, system, mask, ref, ref_mask, mass, device)
    sub = frame_subset(coords.shape[0], frame_indices)
    if sub is None:
        _, moved = superpose_arrays(coords, idx, ref_xyz, w, False, True, device)
        return ArrayTrajectory(moved, box=box, time_ps=time)
    out = coords.copy()
    if sub.size:
        _, moved = superpose_arrays(coords[sub], idx, ref_xyz, w, False, True, device)
        out[sub] = moved
    return ArrayTrajectory(out, box=box, time_ps=time)


__all__ = ["align", "superpose"]
