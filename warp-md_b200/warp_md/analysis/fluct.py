"""``rmsf`` / ``atomicfluct`` / ``bfactors`` with the reference's arguments
(python/warp_md/analysis/fluct.py:149-235): per-atom values as (index, value)
rows, averaged per residue (``byres``, first-seen residue order) or over the
whole mask (``bymask``); ``calcadp`` returns (index, uxx, uyy, uzz, uxy,
uxz, uyz) rows."""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from ..plans import frame_subset, parse_device
from .. import _native as N
from .trajectory import read_all_frames


def _resids(system) -> np.ndarray:
    if hasattr(system, "resids"):
        return np.asarray(system.resids, dtype=np.int64)
    atoms = system.atom_table()
    r = atoms.get("resid", [])
    if not len(r):
        raise ValueError("system atom table has no resid data")
    return np.asarray(r, dtype=np.int64)


def _pack(indices, values) -> np.ndarray:
    idx = np.asarray(indices, dtype=np.int64)
    if idx.size == 0:
        return np.empty((0, 2), dtype=np.float32)
    return np.column_stack((idx.astype(np.float32), np.asarray(values, dtype=np.float64).astype(np.float32)))


def _aggregate(values: np.ndarray, indices: np.ndarray, system, byres: bool, bymask: bool) -> np.ndarray:
    vals = np.asarray(values, dtype=np.float32).reshape(-1)
    idx = np.asarray(indices, dtype=np.int64).reshape(-1)
    if bymask:
        return _pack([0], [float(np.mean(vals)) if vals.size else 0.0])
    if byres:
        res = _resids(system)
        order, groups = [], {}
        for pos, a in enumerate(idx.tolist()):
            if a >= res.size:
                continue
            r = int(res[a])
            if r not in groups:
                groups[r] = []
                order.append(r)
            groups[r].append(pos)
        return _pack(order, [float(np.mean(vals[groups[r]])) for r in order])
    return _pack(idx, vals)


def _indices(system, mask: str) -> np.ndarray:
    sel = system.select(mask if mask else "all")
    return np.asarray(list(sel.indices), dtype=np.int64)


def _moments(traj, system, idx, frame_indices, chunk_frames, want_adp: bool, device: str):
    coords, _b, _t = read_all_frames(traj, chunk_frames)
    if coords is None:
        coords = np.zeros((0, 0, 3), np.float32)
    sub = frame_subset(coords.shape[0], frame_indices)
    if sub is not None:
        coords = coords[sub]
    coords = np.ascontiguousarray(coords, dtype=np.float32)
    n = idx.size
    rmsf = np.zeros(n, np.float32)
    adp = np.zeros((n, 6), np.float32) if want_adp else None
    if n == 0 or coords.shape[0] == 0:
        return rmsf, (np.zeros((0, 6), np.float32) if want_adp else None)
    if int(idx.max()) >= coords.shape[1]:
        raise RuntimeError("invalid selection: selection index out of range")
    ctx = N.context(parse_device(device))
    sel = np.ascontiguousarray(idx, dtype=np.uint32)
    ctx.check(ctx.lib.wmd_rmsf(ctx.handle, coords.ctypes.data, coords.shape[0], coords.shape[1], 3, sel.ctypes.data,
                               n, rmsf.ctypes.data, None if adp is None else adp.ctypes.data, None))
    return rmsf, adp


def rmsf(traj, system, mask: str = "", byres: bool = False, bymask: bool = False, calcadp: bool = False,
         frame_indices: Optional[Sequence[int]] = None, chunk_frames: Optional[int] = None,
         length_scale: float = 1.0, device: str = "auto"):
    """Compute RMSF for selected atoms."""
    if byres and bymask:
        raise ValueError("byres and bymask are mutually exclusive")
    idx = _indices(system, mask)
    if idx.size == 0:
        raise ValueError("selection resolved to empty set")
    if calcadp:
        _, adp = _moments(traj, system, idx, frame_indices, chunk_frames, True, device)
        if adp.size == 0:
            return np.empty((0, 7), dtype=np.float32)
        out = np.empty((adp.shape[0], 7), dtype=np.float32)
        out[:, 0] = idx.astype(np.float32)
        out[:, 1:] = adp * np.float32(length_scale * length_scale)
        return out
    vals, _ = _moments(traj, system, idx, frame_indices, chunk_frames, False, device)
    return _aggregate(vals * np.float32(length_scale), idx, system, byres, bymask)


def atomicfluct(traj, system, mask: str = "", byres: bool = False, bymask: bool = False, calcadp: bool = False,
                frame_indices: Optional[Sequence[int]] = None, chunk_frames: Optional[int] = None,
                length_scale: float = 1.0, device: str = "auto"):
    """Alias of RMSF with optional ADP output."""
    if calcadp and (byres or bymask):
        raise ValueError("calcadp output is only supported for byatom mode")
    return rmsf(traj, system, mask=mask, byres=byres, bymask=bymask, calcadp=calcadp, frame_indices=frame_indices,
                chunk_frames=chunk_frames, length_scale=length_scale, device=device)


def bfactors(traj, system, mask: str = "", byres: bool = True, bymask: bool = False,
             frame_indices: Optional[Sequence[int]] = None, chunk_frames: Optional[int] = None,
             length_scale: float = 1.0, device: str = "auto"):
    """Compute pseudo B-factors from RMSF."""
    if byres and bymask:
        raise ValueError("byres and bymask are mutually exclusive")
    data = rmsf(traj, system, mask=mask, byres=False, bymask=False, frame_indices=frame_indices,
                chunk_frames=chunk_frames, length_scale=length_scale, device=device)
    if data.size == 0:
        return data
    idx = data[:, 0].astype(np.int64)
    v = data[:, 1]
    return _aggregate(8.0 * np.pi * np.pi / 3.0 * v * v, idx, system, byres, bymask)


__all__ = ["rmsf", "atomicfluct", "bfactors"]
