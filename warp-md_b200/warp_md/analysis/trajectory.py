"""In-memory trajectory with the reference's ``read_chunk`` protocol
(python/warp_md/analysis/trajectory.py:13-49): chunks are dicts with
"coords" (frames, atoms, 3) float32 and optional "box" / "time"."""
from __future__ import annotations

from typing import Optional

import numpy as np


class ArrayTrajectory:
    def __init__(self, coords, box: Optional[np.ndarray] = None, time_ps: Optional[np.ndarray] = None):
        self._coords = np.asarray(coords, dtype=np.float32)
        if self._coords.ndim != 3 or self._coords.shape[-1] != 3:
            raise ValueError("coords must be (n_frames, n_atoms, 3)")
        self._box = None if box is None else np.asarray(box, dtype=np.float32)
        self._time = None if time_ps is None else np.asarray(time_ps, dtype=np.float64)
        self._index = 0

    @property
    def coords(self) -> np.ndarray:
        return self._coords

    def reset(self):
        self._index = 0

    def n_atoms(self) -> int:
        return int(self._coords.shape[1])

    def n_frames(self) -> int:
        return int(self._coords.shape[0])

    def read_chunk(self, max_frames: int = 128):
        if self._index >= self._coords.shape[0]:
            return None
        end = min(self._index + max(1, int(max_frames)), self._coords.shape[0])
        chunk = {"coords": self._coords[self._index:end]}
        if self._box is not None:
            chunk["box"] = self._box[self._index:end]
        if self._time is not None:
            chunk["time"] = self._time[self._index:end]
        self._index = end
        return chunk


def read_all_frames(traj, chunk_frames: Optional[int] = None):
    """All frames of a trajectory-like object: our Trajectory / ArrayTrajectory
    (arrays in place) or anything with ``read_chunk`` (read_all_frames,
    python/warp_md/analysis/_runtime.py:638-678).  Returns (coords float32,
    box or None, time or None)."""
    if hasattr(traj, "coords") and not callable(getattr(traj, "coords")):
        coords = np.asarray(traj.coords, dtype=np.float32)
        box = getattr(traj, "box", None) if not isinstance(traj, ArrayTrajectory) else traj._box
        time = getattr(traj, "time_ps", None) if not isinstance(traj, ArrayTrajectory) else traj._time
        return coords, box, time
    if hasattr(traj, "reset"):
        traj.reset()
    parts, boxes, times = [], [], []
    chunk = traj.read_chunk(max(1, int(chunk_frames or 128)))
    while chunk is not None:
        parts.append(np.asarray(chunk["coords"], dtype=np.float32))
        if chunk.get("box") is not None:
            boxes.append(np.asarray(chunk["box"]))
        t = chunk.get("time_ps", chunk.get("time"))
        if t is not None:
            times.append(np.asarray(t))
        chunk = traj.read_chunk(max(1, int(chunk_frames or 128)))
    if not parts:
        return None, None, None
    coords = np.concatenate(parts, axis=0)
    return (coords, np.concatenate(boxes, axis=0) if boxes else None,
            np.concatenate(times, axis=0) if times else None)


__all__ = ["ArrayTrajectory", "read_all_frames"]
