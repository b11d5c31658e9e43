"""Clustering on the GPU (wmd_cluster_dbscan / wmd_cluster_kmeans and
TrajectoryClusterPlan) against the oracle's restatement of the reference's
sequential algorithms.

Parity is exact: DBSCAN labels, sizes and medoids are a function of the float32
matrix, which the FP64 pairwise path reproduces bit for bit in practice; k-means
runs the same FP64 sums in the same order, so labels and sizes agree and a
centroid may differ only between members equidistant from their center.
"""
import numpy as np
import pytest

import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _states(n_atoms, per, seed, spread=1.5):
    """Frames around a few well-separated conformations, plus loners."""
    rng = np.random.default_rng(seed)
    _, ref = synth.make_trajectory(n_atoms, 1, 0.0, seed)
    out = []
    for k, m in enumerate(per):
        base = ref + rng.normal(0, spread, ref.shape).astype(np.float32) * (k > 0)
        fr = base[None] + rng.normal(0, 0.3, (m, n_atoms, 3)).astype(np.float32)
        out.append(fr)
    fr = np.concatenate(out).astype(np.float32)
    rng.shuffle(fr)
    return fr


def _system(n):
    import warp_md

    return warp_md.System.from_arrays({"name": ["CA" if i % 2 == 0 else "X" for i in range(n)],
                                       "resid": list(range(1, n + 1))})


def test_dbscan_plan_matches_oracle():
    import warp_md

    fr = _states(120, [40, 30, 25, 3], 5)
    system = _system(120)
    traj = warp_md.Trajectory.from_numpy(fr)
    for expr in ("all", "name CA"):
        sel = system.select(expr)
        idx = sel.as_array()
        d32, _ = oracle.pairwise(fr[:, idx])
        for eps, ms in ((0.6, 3), (0.45, 5), (1.5, 2), (0.2, 1)):
            out = warp_md.TrajectoryClusterPlan(sel, method="dbscan", eps=eps, min_samples=ms).run(traj, system)
            labels, cent, sizes = oracle.dbscan(d32, eps, ms)
            np.testing.assert_array_equal(out["labels"], labels, err_msg=f"{expr} {eps} {ms}")
            np.testing.assert_array_equal(out["centroids"], cent)
            np.testing.assert_array_equal(out["sizes"], sizes)
            assert out["method"] == "dbscan" and out["n_frames"] == fr.shape[0]


def test_dbscan_chain_and_frame_subset():
    """A long chain of near neighbours (one cluster through many unions) and a
    frame subset."""
    import warp_md

    rng = np.random.default_rng(2)
    _, ref = synth.make_trajectory(60, 1, 0.0, 9)
    steps = rng.normal(0, 0.05, (300, 60, 3)).astype(np.float32)
    fr = (ref[None] + np.cumsum(steps, axis=0)).astype(np.float32)
    system = _system(60)
    traj = warp_md.Trajectory.from_numpy(fr)
    sel = system.select("all")
    d32, _ = oracle.pairwise(fr)
    out = warp_md.TrajectoryClusterPlan(sel, eps=0.12, min_samples=2).run(traj, system)
    labels, cent, sizes = oracle.dbscan(d32, 0.12, 2)
    np.testing.assert_array_equal(out["labels"], labels)
    np.testing.assert_array_equal(out["centroids"], cent)
    np.testing.assert_array_equal(out["sizes"], sizes)
    sub = [5, -1, 40, 7, 7]
    out = warp_md.TrajectoryClusterPlan(sel, eps=0.5, min_samples=1).run(traj, system, frame_indices=sub)
    idx = np.array([5, 299, 40, 7, 7])
    d32, _ = oracle.pairwise(fr[idx])
    labels, cent, sizes = oracle.dbscan(d32, 0.5, 1)
    np.testing.assert_array_equal(out["labels"], labels)


def test_dbscan_medoid_with_near_duplicate_frames():
    """Near-duplicate frames give distances of ~1e-7 A next to ~1 A ones, so
    the medoid sums take the sequential path (the lanes' partial sums could
    round); labels, sizes and medoids still match the oracle exactly."""
    import warp_md

    rng = np.random.default_rng(4)
    _, ref = synth.make_trajectory(40, 1, 0.0, 2)
    base = ref[None] + rng.normal(0, 0.4, (60, 40, 3)).astype(np.float32)
    dup = base[:20] + np.float32(1e-6) * rng.standard_normal((20, 40, 3)).astype(np.float32)
    fr = np.concatenate([base, dup]).astype(np.float32)
    system = _system(40)
    traj = warp_md.Trajectory.from_numpy(fr)
    sel = system.select("all")
    d32, _ = oracle.pairwise(fr)
    assert d32[d32 > 0].min() < 1e-5
    for eps, ms in ((1.2, 3), (0.8, 2)):
        out = warp_md.TrajectoryClusterPlan(sel, eps=eps, min_samples=ms).run(traj, system)
        labels, cent, sizes = oracle.dbscan(d32, eps, ms)
        np.testing.assert_array_equal(out["labels"], labels)
        np.testing.assert_array_equal(out["centroids"], cent)
        np.testing.assert_array_equal(out["sizes"], sizes)


def test_kmeans_plan_matches_oracle():
    import warp_md

    fr = _states(80, [25, 25, 20, 2], 7)
    system = _system(80)
    traj = warp_md.Trajectory.from_numpy(fr)
    for expr, k, seed in (("all", 3, 0), ("name CA", 4, 123), ("all", 1, 5), ("all", 9, 77)):
        sel = system.select(expr)
        out = warp_md.TrajectoryClusterPlan(sel, method="kmeans", n_clusters=k, seed=seed).run(traj, system)
        labels, cent, sizes = oracle.kmeans(fr, selection=sel.as_array(), n_clusters=k, seed=seed)
        np.testing.assert_array_equal(out["labels"], labels, err_msg=f"{expr} {k} {seed}")
        np.testing.assert_array_equal(out["sizes"], sizes)
        _check_centroids(out["centroids"], cent, labels, _features(fr, sel.as_array()))
        assert out["method"] == "kmeans"


def _features(fr, idx):
    """build_aligned_features in numpy: each frame's selection onto frame 0's."""
    y = fr[0][idx].astype(np.float64)
    cy = y.mean(0)
    out = []
    for f in range(fr.shape[0]):
        x = fr[f][idx].astype(np.float64)
        cx = x.mean(0)
        u, _s, vt = np.linalg.svd((x - cx).T @ (y - cy))
        r = vt.T @ u.T
        if np.linalg.det(r) < 0:
            vt[-1] *= -1
            r = vt.T @ u.T
        out.append(((x - cx) @ r.T + cy).reshape(-1))
    return np.array(out)


def _check_centroids(got, want, labels, feat):
    """Centroids agree, except where two members are equidistant from the
    center (a two-member cluster's midpoint, say): then FP64 rounding, not the
    algorithm, picks the member, and both are accepted."""
    for c, (g, w) in enumerate(zip(got, want)):
        if g == w:
            continue
        mem = labels == c
        center = feat[mem].mean(0)
        dg = ((feat[g] - center) ** 2).sum()
        dw = ((feat[w] - center) ** 2).sum()
        assert labels[g] == c and abs(dg - dw) <= 1e-9 * max(dg, dw, 1e-30), (c, g, w, dg, dw)


def test_cluster_errors_and_empty():
    import warp_md

    fr = _states(20, [5], 1)
    system = _system(20)
    traj = warp_md.Trajectory.from_numpy(fr)
    sel = system.select("all")
    with pytest.raises(RuntimeError, match="eps must be > 0"):
        warp_md.TrajectoryClusterPlan(sel, eps=0.0).run(traj, system)
    with pytest.raises(RuntimeError, match="memory_budget_bytes"):
        warp_md.TrajectoryClusterPlan(sel, memory_budget_bytes=8).run(traj, system)
    with pytest.raises(RuntimeError, match="non-empty selection"):
        warp_md.TrajectoryClusterPlan(system.select_indices([])).run(traj, system)
    out = warp_md.TrajectoryClusterPlan(sel).run(warp_md.Trajectory.from_numpy(fr[:0]), system)
    assert out["n_frames"] == 0 and out["labels"].size == 0
