"""``cluster_trajectory`` with the reference's arguments
(python/warp_md/analysis/clustering.py:76-141): the mask (an expression, or
atom indices) selects the atoms, then TrajectoryClusterPlan runs DBSCAN or
k-means; the result dict has numpy arrays."""
from __future__ import annotations

from typing import Any, Optional, Sequence, Union

import numpy as np

MaskLike = Union[str, Sequence[int], np.ndarray]


_WHOLE_SYSTEM = frozenset({"", "*", "all"})


def _whole_system_expression(system) -> str:
    """The expression a blank mask stands for: every residue, written as the
    closed resid range of the system's atom table (``all`` for a system that
    has no table, ``resid 0:0`` for an empty one)."""
    table = system.atom_table() if hasattr(system, "atom_table") else None
    if table is None:
        return "all"
    ids = np.asarray(table.get("resid", []), dtype=np.int64).reshape(-1)
    lo, hi = (int(ids.min()), int(ids.max())) if ids.size else (0, 0)
    return "resid %d:%d" % (lo, hi)


def _selection_for(system, mask: MaskLike):
    """A string mask is a selection expression (blank, ``*`` and ``all``
    mean the whole system, as does None); anything else is a list of atom
    indices, which the system must accept through ``select_indices``."""
    if mask is None or isinstance(mask, str):
        text = "" if mask is None else mask
        return system.select(_whole_system_expression(system) if text in _WHOLE_SYSTEM else text)
    by_index = getattr(system, "select_indices", None)
    if by_index is None:
        raise RuntimeError("an index mask needs a system with select_indices(); this one has none")
    return by_index([int(i) for i in np.asarray(mask, dtype=np.int64).ravel()])


def cluster_trajectory(traj, system, mask: MaskLike = "", method: str = "dbscan", eps: float = 2.0,
                       min_samples: int = 5, n_clusters: int = 8, max_iter: int = 100, tol: float = 1.0e-4,
                       seed: int = 0, frame_indices: Optional[Sequence[int]] = None,
                       chunk_frames: Optional[int] = None, device: str = "auto",
                       memory_budget_bytes: Optional[int] = None) -> dict[str, Any]:
    """Cluster trajectory frames using DBSCAN or KMeans on RMSD-aligned coordinates."""
    m = str(method).strip().lower()
    if m not in ("dbscan", "kmeans"):
        raise ValueError("method must be 'dbscan' or 'kmeans'")
    import warp_md

    plan = warp_md.TrajectoryClusterPlan(_selection_for(system, mask), method=m, eps=float(eps),
                                         min_samples=int(min_samples), n_clusters=int(n_clusters),
                                         max_iter=int(max_iter), tol=float(tol), seed=int(seed),
                                         memory_budget_bytes=memory_budget_bytes)
    out = plan.run(traj, system, chunk_frames=chunk_frames, device=device,
                   frame_indices=None if frame_indices is None else [int(v) for v in frame_indices])
    if not isinstance(out, dict):
        raise RuntimeError("TrajectoryClusterPlan returned unexpected output type")
    return {"labels": np.asarray(out.get("labels", []), dtype=np.int32),
            "centroids": np.asarray(out.get("centroids", []), dtype=np.uint32),
            "sizes": np.asarray(out.get("sizes", []), dtype=np.uint32),
            "method": out.get("method", m), "n_frames": int(out.get("n_frames", 0))}


__all__ = ["cluster_trajectory"]
