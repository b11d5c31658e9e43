"""DCD trajectories read through the GPU decoder (``Trajectory.open_dcd``).

Mirrors the reference's ``PyTrajectory.open_dcd`` / ``read_chunk`` /
``reset`` / ``count_frames`` (crates/traj-py/src/io.rs:687-708, 1335-1571)
over ``DcdReader`` (crates/traj-io/src/dcd.rs).  The library parses the
header on the host, preads raw frame bytes into pinned buffers with several
threads and decodes them on the GPU (record markers, byte order, atom
selection, length scale); unit cells are decoded on the host.  ``RmsdPlan``
runs on a DCD trajectory without a host copy of the frames
(``wmd_dcd_rmsd``: the file read, the copy and the kernels overlap).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .core import System, Trajectory

# heuristic_chunk_frames (crates/traj-py/src/pack.rs:1360-1362, 1447-1466)
_AUTO_CHUNK_MIN, _AUTO_CHUNK_MAX, _AUTO_CHUNK_TARGET_BYTES = 16, 256, 8 * 1024 * 1024


def heuristic_chunk_frames(n_atoms: int) -> int:
    per_frame = n_atoms * 16
    if per_frame == 0:
        return 64
    raw = min(max(_AUTO_CHUNK_TARGET_BYTES // per_frame, _AUTO_CHUNK_MIN), _AUTO_CHUNK_MAX)
    p = 1
    while p < raw:
        p <<= 1
    lower, upper = p >> 1, p
    chunk = lower if (lower >= _AUTO_CHUNK_MIN and raw - lower <= upper - raw) else upper
    return min(max(chunk, _AUTO_CHUNK_MIN), _AUTO_CHUNK_MAX)


def _box_arrays(kinds: np.ndarray, mats: np.ndarray, include_box: bool, include_box_matrix: bool):
    """Box / box_matrix outputs of read_chunk (io.rs:1463-1514): lengths only
    when every frame is orthorhombic, matrices when no frame lacks a box."""
    if kinds.size == 0 or np.any(kinds == 0):
        return None, None
    box = mats[:, [0, 4, 8]].copy() if include_box and np.all(kinds == 1) else None
    mat = mats.reshape(-1, 3, 3).copy() if include_box_matrix else None
    return box, mat


class DcdTrajectory(Trajectory):
    """A DCD file on one CUDA device.  ``coords`` (every frame, host memory) is
    read on first use, for plans that take whole arrays."""

    def __init__(self, path: str, system: System, length_scale: Optional[float] = None, device: int = 0):
        self.ctx = N.context(device)
        self.path = str(path)
        self.length_scale = 1.0 if length_scale is None else float(length_scale)
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.wmd_dcd_open(self.ctx.handle, self.path.encode(), self.length_scale,
                                                 ctypes.byref(h)))
        self.handle = h
        na, nf, hf = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.ctx.lib.wmd_dcd_info(self.handle, ctypes.byref(na), ctypes.byref(nf), ctypes.byref(hf))
        self._n_atoms, self._header_frames = na.value, hf.value
        if self._n_atoms != system.n_atoms():
            self.close()
            raise RuntimeError("trajectory atom count does not match system")
        self._cursor = 0
        self._coords: Optional[np.ndarray] = None
        self._box: Optional[np.ndarray] = None
        self.time_ps = None

    # -- reference surface -------------------------------------------------
    def n_atoms(self) -> int:
        return self._n_atoms

    def n_frames(self) -> int:
        return self._frames()

    def n_frames_hint(self) -> Optional[int]:
        return self._header_frames or None

    def count_frames(self, chunk_frames: Optional[int] = None) -> int:
        return self._frames()

    def reset(self) -> None:
        self._cursor = 0

    def skip_frames(self, n: int) -> int:
        k = max(0, min(int(n), self._frames() - self._cursor))
        self._cursor += k
        return k

    def read_chunk(self, max_frames: Optional[int] = None, include_box: bool = True, include_box_matrix: bool = True,
                   include_time: bool = True, atom_indices: Optional[Sequence[int]] = None,
                   include_velocities: bool = False, include_forces: bool = False, include_lambda: bool = False):
        """Next chunk from the cursor as the reference's dict, or None at the end."""
        if atom_indices is not None and len(atom_indices) == 0:
            raise RuntimeError("atom_indices must not be empty")
        n_out = self._n_atoms if atom_indices is None else len(atom_indices)
        if max_frames is None:
            max_frames = heuristic_chunk_frames(n_out if atom_indices is not None else self._n_atoms)
        max_frames = max(1, int(max_frames))
        coords, kinds, mats = self._read(self._cursor, max_frames, atom_indices, include_box or include_box_matrix)
        n = coords.shape[0]
        self._cursor += n
        if n == 0:
            return None
        box, mat = _box_arrays(kinds, mats, include_box, include_box_matrix)
        return {"coords": coords, "box": box, "box_matrix": mat, "time_ps": None, "velocities": None,
                "forces": None, "lambda_value": None, "frames": n}

    def read_frames(self, frame_indices: Sequence[int], chunk_frames: Optional[int] = None, include_box: bool = True,
                    include_box_matrix: bool = True, include_time: bool = False, **_unused):
        """Frames by index (negative indices count from the end)."""
        nf = self._frames()
        idx = [int(i) + nf if int(i) < 0 else int(i) for i in frame_indices]
        idx = [i for i in idx if 0 <= i < nf]
        if not idx:
            return None
        parts = [self._read(i, 1, None, include_box or include_box_matrix) for i in idx]
        coords = np.concatenate([p[0] for p in parts])
        kinds = np.concatenate([p[1] for p in parts])
        mats = np.concatenate([p[2] for p in parts])
        box, mat = _box_arrays(kinds, mats, include_box, include_box_matrix)
        return {"coords": coords, "box": box, "box_matrix": mat, "time_ps": None, "frames": len(idx),
                "source_indices": np.asarray(idx, np.int64)}

    # -- whole-array access for the plans ----------------------------------
    @property
    def coords(self) -> np.ndarray:
        if self._coords is None:
            parts, kinds, mats, pos = [], [], [], 0
            step = max(1, (1 << 30) // max(1, self._n_atoms * 12))
            while True:
                c, k, m = self._read(pos, step, None, True)
                if c.shape[0] == 0:
                    break
                parts.append(c)
                kinds.append(k)
                mats.append(m)
                pos += c.shape[0]
            self._coords = np.concatenate(parts) if parts else np.zeros((0, self._n_atoms, 3), np.float32)
            if parts:
                self._box, _ = _box_arrays(np.concatenate(kinds), np.concatenate(mats), True, False)
        return self._coords

    def read_device(self, first: int, n: int, atom_indices=None, out=None):
        """Frames [first, first + n) decoded into a CUDA tensor (torch)."""
        import torch

        n_out = self._n_atoms if atom_indices is None else len(atom_indices)
        n = max(0, min(int(n), self._frames() - int(first)))
        if out is None:
            out = torch.empty((n, n_out, 3), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        sel = None if atom_indices is None else np.ascontiguousarray(atom_indices, np.uint32)
        got = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.wmd_dcd_read(self.ctx.handle, self.handle, int(first), n, N.ptr(sel),
                                                 0 if sel is None else sel.size, out.data_ptr(), None, None,
                                                 ctypes.byref(got), torch.cuda.current_stream().cuda_stream))
        return out[: got.value]

    def rmsd(self, ref: np.ndarray, atom_indices=None, align: bool = True, first: int = 0,
             n: Optional[int] = None) -> np.ndarray:
        """Per-frame RMSD of frames [first, first + n) straight from the file."""
        total = self._frames() - int(first)
        n = total if n is None else max(0, min(int(n), total))
        sel = None if atom_indices is None else np.ascontiguousarray(atom_indices, np.uint32)
        r = N.Reference.from_numpy(self.ctx, ref)
        try:
            out = np.empty(max(n, 0), np.float64)
            got = ctypes.c_int64()
            self.ctx.check(self.ctx.lib.wmd_dcd_rmsd(self.ctx.handle, self.handle, int(first), max(n, 0), N.ptr(sel),
                                                     0 if sel is None else sel.size, r.handle, int(align),
                                                     out.ctypes.data, ctypes.byref(got), None))
        finally:
            r.close()
        return out[: got.value]

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx.lib.wmd_dcd_close(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def box(self) -> Optional[np.ndarray]:
        """Per-frame orthorhombic box lengths (frames, 3), float32, when every
        frame carries an orthorhombic unit cell; otherwise None.  Read with
        ``coords``."""
        if self._coords is None:
            self.coords
        return self._box

    # -- internals -----------------------------------------------------------
    def _frames(self) -> int:
        na, nf, hf = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self.ctx.lib.wmd_dcd_info(self.handle, ctypes.byref(na), ctypes.byref(nf), ctypes.byref(hf))
        return nf.value

    def _read(self, first: int, max_frames: int, atom_indices, want_box: bool):
        n_out = self._n_atoms if atom_indices is None else len(atom_indices)
        cap = max(0, min(max_frames, self._frames() - first))
        sel = None if atom_indices is None else np.ascontiguousarray(np.asarray(atom_indices, np.int64), np.uint32)
        coords = np.empty((cap, n_out, 3), np.float32)
        kinds = np.zeros(cap, np.int32)
        mats = np.zeros((cap, 9), np.float32)
        got = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.wmd_dcd_read(self.ctx.handle, self.handle, int(first), int(max_frames), N.ptr(sel),
                                                 0 if sel is None else sel.size, coords.ctypes.data if cap else None,
                                                 kinds.ctypes.data if want_box and cap else None,
                                                 mats.ctypes.data if want_box and cap else None, ctypes.byref(got),
                                                 None))
        k = got.value
        return coords[:k], kinds[:k], mats[:k]


def open_dcd(path: str, system: System, length_scale: Optional[float] = None, device: int = 0) -> DcdTrajectory:
    return DcdTrajectory(path, system, length_scale, device)
