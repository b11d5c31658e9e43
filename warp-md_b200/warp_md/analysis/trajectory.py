"""In-memory trajectory with the reference's ``read_chunk`` protocol
(python/warp_md/analysis/trajectory.py:13-49): chunks are dicts with
"coords" (frames, atoms, 3) float32 and optional "box" / "time"."""
from __future__ import annotations

from typing import Optional

import numpy as np


class ArrayTrajectory:
    """Frames held in memory behind the chunked reader protocol: a cursor
    walks the frames, and each ``read_chunk`` hands out the next slice as a
    dict ("coords" always; "box" and "time" when given), None at the end.
    Arrays are kept as float32 coordinates and box, float64 times."""

    def __init__(self, coords, box: Optional[np.ndarray] = None, time_ps: Optional[np.ndarray] = None):
        frames = np.asarray(coords, dtype=np.float32)
        if frames.ndim != 3 or frames.shape[2] != 3:
            raise ValueError(f"ArrayTrajectory needs coordinates shaped (frames, atoms, 3); got {frames.shape}")
        self.frames = frames
        self.box_values = None if box is None else np.asarray(box, dtype=np.float32)
        self.time_values = None if time_ps is None else np.asarray(time_ps, dtype=np.float64)
        self.cursor = 0

    @property
    def coords(self) -> np.ndarray:
        return self.frames

    def n_frames(self) -> int:
        return self.frames.shape[0]

    def n_atoms(self) -> int:
        return self.frames.shape[1]

    def reset(self):
        self.cursor = 0

    def read_chunk(self, max_frames: int = 128):
        lo = self.cursor
        if lo >= self.n_frames():
            return None
        hi = min(self.n_frames(), lo + max(int(max_frames), 1))
        self.cursor = hi
        chunk = {"coords": self.frames[lo:hi]}
        for key, values in (("box", self.box_values), ("time", self.time_values)):
            if values is not None:
                chunk[key] = values[lo:hi]
        return chunk


def read_all_frames(traj, chunk_frames: Optional[int] = None):
    """All frames of a trajectory-like object: our Trajectory / ArrayTrajectory
    (arrays in place) or anything with ``read_chunk`` (read_all_frames,
    python/warp_md/analysis/_runtime.py:638-678).  Returns (coords float32,
    box or None, time or None)."""
    if hasattr(traj, "coords") and not callable(getattr(traj, "coords")):
        coords = np.asarray(traj.coords, dtype=np.float32)
        if isinstance(traj, ArrayTrajectory):
            return coords, traj.box_values, traj.time_values
        box = getattr(traj, "box", None)
        time = getattr(traj, "time_ps", None)
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
