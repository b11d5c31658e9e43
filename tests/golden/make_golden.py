"""Generates tests/golden/rmsd_golden.npz from the reference's own numpy Kabsch
helpers.

Run in a container where the warp-md reference checkout is available:

    python tests/golden/make_golden.py /path/to/warp-md/python

The script imports ``warp_md.analysis._runtime.kabsch_rmsd`` and ``rmsd_raw``
(python/warp_md/analysis/_runtime.py:611-635 in warp-md 0.4.30) -- FP64 numpy
SVD Kabsch with explicit residuals, the same algorithm as
crates/traj-engine/src/plans/rmsd/plan.rs:1161-1248 -- in a subprocess whose
PYTHONPATH points at that checkout, so the reference package never shadows
this repository's ``warp_md``.  The fixtures are small seeded cases; the test
suite checks the C oracle against them.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "warp-md_b200"))

from warp_md import synth  # noqa: E402

CHILD = r"""
import sys, json, numpy as np
from warp_md.analysis._runtime import kabsch_rmsd, rmsd_raw
d = np.load(sys.argv[1])
out = {}
for key in d.files:
    if not key.startswith("frames_"):
        continue
    name = key[len("frames_"):]
    frames = d[key].astype(np.float64)
    ref = d["ref_" + name].astype(np.float64)
    out["aligned_" + name] = [kabsch_rmsd(f, ref) for f in frames]
    out["raw_" + name] = [rmsd_raw(f, ref) for f in frames]
    if frames.shape[0] <= 24:
        n = frames.shape[0]
        m = np.zeros((n, n)); r = np.zeros((n, n))
        for i in range(n):
            for j in range(i + 1, n):
                m[i, j] = m[j, i] = kabsch_rmsd(frames[i], frames[j])
                r[i, j] = r[j, i] = rmsd_raw(frames[i], frames[j])
        out["pair_aligned_" + name] = m.tolist()
        out["pair_raw_" + name] = r.tolist()
json.dump(out, open(sys.argv[2], "w"))
"""


def cases():
    c = {}
    # config-0 recipe at small sizes
    for n_atoms, n_frames, sigma, seed in [(3, 8, 0.5, 1), (31, 12, 0.5, 2), (257, 16, 0.5, 3),
                                          (1000, 10, 0.05, 4), (3000, 6, 0.5, 5)]:
        fr, ref = synth.make_trajectory(n_atoms, n_frames, sigma, seed)
        c[f"walk_{n_atoms}"] = (fr, ref)
    # noise levels spanning the streaming workload's range
    fr, ref = synth.make_trajectory(2048, 12, (0.05, 3.0), 6)
    c["walk_2048_sigmarange"] = (fr, ref)
    # drifting trajectory (pairwise workload recipe)
    fr = synth.make_drift_trajectory(200, 16, 0.1, 7)
    c["drift_200"] = (fr, fr[0].copy())
    # degenerate geometries: collinear and planar structures
    rng = np.random.default_rng(8)
    line = np.zeros((20, 3)); line[:, 0] = np.arange(20) * 1.5
    fr = np.stack([line @ synth.haar_rotation(rng).T + rng.normal(0, 5, 3) + rng.normal(0, 0.2, line.shape)
                   for _ in range(6)]).astype(np.float32)
    c["collinear_20"] = (fr, line.astype(np.float32))
    plane = np.zeros((40, 3)); plane[:, :2] = rng.normal(0, 6, (40, 2))
    fr = np.stack([plane @ synth.haar_rotation(rng).T + rng.normal(0, 5, 3) + rng.normal(0, 0.3, plane.shape)
                   for _ in range(6)]).astype(np.float32)
    c["planar_40"] = (fr, plane.astype(np.float32))
    # mirrored structure (forces the reflection fix)
    fr0, ref0 = synth.make_trajectory(50, 4, 0.1, 9)
    mir = fr0.copy(); mir[:, :, 2] *= -1
    c["mirror_50"] = (mir, ref0)
    return c


def main(ref_python: str) -> None:
    data = {}
    for name, (fr, ref) in cases().items():
        data["frames_" + name] = fr.astype(np.float32)
        data["ref_" + name] = ref.astype(np.float32)
    tmp_in = os.path.join(HERE, "_inputs_tmp.npz")
    tmp_out = os.path.join(HERE, "_outputs_tmp.json")
    np.savez(tmp_in, **data)
    env = dict(os.environ, PYTHONPATH=ref_python)
    subprocess.run([sys.executable, "-c", CHILD, tmp_in, tmp_out], check=True, env=env, cwd="/tmp")
    res = json.load(open(tmp_out))
    for k, v in res.items():
        data["expect_" + k] = np.asarray(v, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "rmsd_golden.npz"), **data)
    os.remove(tmp_in)
    os.remove(tmp_out)
    print("wrote", os.path.join(HERE, "rmsd_golden.npz"), "with", len(data), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference's python/ directory>")
    main(sys.argv[1])
