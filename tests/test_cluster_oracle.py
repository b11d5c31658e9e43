"""The oracle's clustering (TrajectoryClusterPlan: DBSCAN, k-means) against an
independent Python transcription of the reference's loops
(crates/traj-engine/src/plans/analysis/clustering.rs:269-548), and the
cluster_trajectory wrapper's argument passing (the reference's
test_cluster_trajectory_uses_plan, with a stand-in plan), on the CPU."""
from collections import deque

import numpy as np

import oracle


def _py_dbscan(D, eps, min_samples):
    n = D.shape[0]
    d = lambda i, j: 0.0 if i == j else float(D[i, j])  # noqa: E731
    labels = [-2] * n
    visited = [False] * n
    cid = 0
    for i in range(n):
        if visited[i]:
            continue
        visited[i] = True
        neigh = [j for j in range(n) if d(i, j) <= eps]
        if len(neigh) < min_samples:
            labels[i] = -1
            continue
        labels[i] = cid
        queued = [False] * n
        q = deque()
        for p in neigh:
            if p != i and not queued[p]:
                q.append(p)
                queued[p] = True
        while q:
            p = q.popleft()
            if not visited[p]:
                visited[p] = True
                nb = [j for j in range(n) if d(p, j) <= eps]
                if len(nb) >= min_samples:
                    for r in nb:
                        if not queued[r]:
                            q.append(r)
                            queued[r] = True
            if labels[p] in (-2, -1):
                labels[p] = cid
        cid += 1
    cent, sizes = [], []
    for c in range(cid):
        mem = [i for i in range(n) if labels[i] == c]
        sizes.append(len(mem))
        best, bs = mem[0], np.inf
        for a in mem:
            s = 0.0
            for b in mem:
                s += d(a, b)
            if s < bs:
                bs, best = s, a
        cent.append(best)
    return np.array(labels, np.int32), np.array(cent, np.uint32), np.array(sizes, np.uint32)


def test_dbscan_matches_transcription():
    rng = np.random.default_rng(0)
    for trial in range(12):
        n = int(rng.integers(5, 60))
        pts = np.concatenate([rng.normal(c, 0.4, (n // 3 + 1, 2)) for c in rng.uniform(-5, 5, (3, 2))])[:n]
        D = np.sqrt(((pts[:, None] - pts[None]) ** 2).sum(-1)).astype(np.float32)
        eps = float(np.float32(rng.uniform(0.2, 1.2)))
        ms = int(rng.integers(1, 6))
        got = oracle.dbscan(D, eps, ms)
        want = _py_dbscan(D, eps, ms)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


def test_kmeans_is_deterministic_and_complete():
    from warp_md import synth

    fr, _ = synth.make_trajectory(30, 40, 0.5, 3)
    fr[10:20] += np.random.default_rng(1).normal(0, 2, (10, 30, 3)).astype(np.float32)
    a = oracle.kmeans(fr, n_clusters=4, seed=11)
    b = oracle.kmeans(fr, n_clusters=4, seed=11)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    labels, cent, sizes = a
    assert sizes.sum() == 40 and len(cent) == 4
    for c in range(4):
        assert sizes[c] == (labels == c).sum()
        if sizes[c]:
            assert labels[cent[c]] == c


def test_cluster_trajectory_passes_arguments(monkeypatch):
    """test_cluster_trajectory_uses_plan of the reference (python/warp_md/tests/test_clustering.py)."""
    import warp_md
    from warp_md.analysis.clustering import cluster_trajectory

    called = {}

    class _Sel:
        def __init__(self, indices):
            self.indices = indices

    class _Sys:
        def atom_table(self):
            return {"resid": [1, 2, 3, 4]}

        def select(self, _mask):
            return _Sel(range(4))

        def select_indices(self, indices):
            return _Sel(indices)

    class _Plan:
        def __init__(self, sel, method="dbscan", eps=2.0, min_samples=5, n_clusters=8, max_iter=100, tol=1.0e-4,
                     seed=0, memory_budget_bytes=None):
            called.update(selection=list(sel.indices), method=method, eps=eps, min_samples=min_samples,
                          n_clusters=n_clusters, max_iter=max_iter, tol=tol, seed=seed,
                          memory_budget_bytes=memory_budget_bytes)

        def run(self, _traj, _system, chunk_frames=None, device="auto", frame_indices=None):
            called.update(chunk_frames=chunk_frames, device=device, frame_indices=frame_indices)
            return {"labels": [0, 0, -1], "centroids": [0], "sizes": [2], "method": "dbscan", "n_frames": 3}

    monkeypatch.setattr(warp_md, "TrajectoryClusterPlan", _Plan, raising=False)
    out = cluster_trajectory(object(), _Sys(), mask=[0, 2, 3], method="dbscan", eps=1.5, min_samples=2,
                             frame_indices=[1, -1], chunk_frames=64, device="cuda", memory_budget_bytes=1024)
    assert called == {"selection": [0, 2, 3], "method": "dbscan", "eps": 1.5, "min_samples": 2, "n_clusters": 8,
                      "max_iter": 100, "tol": 1.0e-4, "seed": 0, "memory_budget_bytes": 1024, "chunk_frames": 64,
                      "device": "cuda", "frame_indices": [1, -1]}
    np.testing.assert_array_equal(out["labels"], np.array([0, 0, -1], dtype=np.int32))
    np.testing.assert_array_equal(out["centroids"], np.array([0], dtype=np.uint32))
    np.testing.assert_array_equal(out["sizes"], np.array([2], dtype=np.uint32))
    assert out["method"] == "dbscan" and out["n_frames"] == 3
