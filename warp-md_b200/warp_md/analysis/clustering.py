"""``cluster_trajectory`` with the reference's arguments
(python/warp_md/analysis/clustering.py:76-141): the mask (an expression, or
atom indices) selects the atoms, then TrajectoryClusterPlan runs DBSCAN or
k-means; the result dict has numpy arrays."""
from __future__ import annotations

from typing import Any, Optional, Sequence, Union

import numpy as np

MaskLike = Union[str, Sequence[int], np.ndarray]


def _all_resid_mask(system) -> str:
    if not hasattr(system, "atom_table"):
        return "all"
    resids = system.atom_table().get("resid", [])
    if not len(resids):
        return "resid 0:0"
    return f"resid {min(resids)}:{max(resids)}"


def _select(system, mask: MaskLike):
    if isinstance(mask, str):
        expr = mask if mask not in ("", "*", "all", None) else _all_resid_mask(system)
        return system.select(expr)
    indices = np.asarray(mask, dtype=np.int64).reshape(-1).tolist()
    if hasattr(system, "select_indices"):
        return system.select_indices(indices)
    raise RuntimeError("system does not support index-based selection (missing select_indices)")


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

    plan = warp_md.TrajectoryClusterPlan(_select(system, mask), method=m, eps=float(eps),
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
