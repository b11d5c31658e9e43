"""Seeded synthetic trajectories with the shapes and value distributions of the
RMSD benchmark workloads (no trajectory files travel with this library).

* reference structure: a 3D random walk with 3.8 A steps along isotropic
  directions (normalised Gaussian 3-vectors), first atom at the origin;
* a frame: ``R_haar @ ref + t + eps`` with R a uniform random rotation (unit
  quaternion from four Gaussians), ``t ~ N(0, 10 A)`` per axis and
  ``eps ~ N(0, sigma^2)`` per atom and axis;
* a drifting trajectory (all-pairs workload): ``frame_{t+1} = frame_t +
  N(0, 0.1 A)`` per atom, each stored frame then under its own random rigid
  motion.

The numpy generators use PCG64 and are the ones tests use.  ``*_torch``
variants build the multi-GB workloads directly in device memory with torch's
generator; they follow the same recipe but not the same random stream.
"""
from __future__ import annotations

from typing import Sequence, Tuple, Union

import numpy as np

Sigma = Union[float, Tuple[float, float]]


def random_walk(n_atoms: int, rng: np.random.Generator, step: float = 3.8) -> np.ndarray:
    d = rng.standard_normal((n_atoms, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[0] = 0.0
    return np.cumsum(step * d, axis=0)


def haar_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    return quat_to_matrix(q)


def quat_to_matrix(q: Sequence[float]) -> np.ndarray:
    w, x, y, z = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
        ]
    )


def make_trajectory(
    n_atoms: int,
    n_frames: int,
    sigma: Sigma = 0.5,
    seed: int = 0,
    trans_sigma: float = 10.0,
) -> Tuple[np.ndarray, np.ndarray]:
    """Returns (coords float32 [n_frames, n_atoms, 3], reference float32 [n_atoms, 3]).
    ``sigma`` is a fixed noise level or a (lo, hi) range drawn per frame."""
    rng = np.random.default_rng(seed)
    ref = random_walk(n_atoms, rng)
    out = np.empty((n_frames, n_atoms, 3), np.float32)
    for f in range(n_frames):
        s = sigma if np.isscalar(sigma) else rng.uniform(sigma[0], sigma[1])
        r = haar_rotation(rng)
        t = rng.normal(0.0, trans_sigma, 3)
        out[f] = ref @ r.T + t + rng.normal(0.0, s, (n_atoms, 3))
    return out, ref.astype(np.float32)


def make_drift_trajectory(
    n_atoms: int, n_frames: int, step_sigma: float = 0.1, seed: int = 0, trans_sigma: float = 10.0
) -> np.ndarray:
    """All-pairs workload: slow random drift, each frame under a random rigid motion."""
    rng = np.random.default_rng(seed)
    cur = random_walk(n_atoms, rng)
    out = np.empty((n_frames, n_atoms, 3), np.float32)
    for f in range(n_frames):
        if f:
            cur = cur + rng.normal(0.0, step_sigma, cur.shape)
        r = haar_rotation(rng)
        out[f] = cur @ r.T + rng.normal(0.0, trans_sigma, 3)
    return out


# ---------------------------------------------------------------------------
# device-side builders for the multi-GB workloads
# ---------------------------------------------------------------------------

def _torch_haar(n: int, gen, device):
    import torch

    q = torch.randn(n, 4, generator=gen, device=device, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    r = torch.stack(
        [
            1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
            2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
            2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
        ],
        dim=1,
    ).reshape(n, 3, 3)
    return r


def make_trajectory_torch(
    n_atoms: int,
    n_frames: int,
    sigma: Sigma = 0.5,
    seed: int = 0,
    device="cuda",
    trans_sigma: float = 10.0,
    chunk: int = 256,
    out=None,
):
    """Device-resident version of :func:`make_trajectory`, built in frame chunks
    so that the temporary memory stays a few hundred MB."""
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    d = torch.randn(n_atoms, 3, generator=gen, device=device, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    d[0] = 0
    ref = torch.cumsum(3.8 * d, dim=0)
    if out is None:
        out = torch.empty(n_frames, n_atoms, 3, device=device, dtype=torch.float32)
    for f0 in range(0, n_frames, chunk):
        f1 = min(n_frames, f0 + chunk)
        m = f1 - f0
        if np.isscalar(sigma):
            s = torch.full((m, 1, 1), float(sigma), device=device, dtype=torch.float64)
        else:
            s = (sigma[0] + (sigma[1] - sigma[0]) * torch.rand(m, 1, 1, generator=gen, device=device,
                                                                dtype=torch.float64))
        r = _torch_haar(m, gen, device)
        t = trans_sigma * torch.randn(m, 1, 3, generator=gen, device=device, dtype=torch.float64)
        blk = torch.matmul(ref.unsqueeze(0), r.transpose(1, 2)) + t
        blk += s * torch.randn(m, n_atoms, 3, generator=gen, device=device, dtype=torch.float64)
        out[f0:f1] = blk.to(torch.float32)
    return out, ref.to(torch.float32)


def make_drift_trajectory_torch(n_atoms: int, n_frames: int, step_sigma: float = 0.1, seed: int = 0,
                                device="cuda", trans_sigma: float = 10.0, chunk: int = 512):
    import torch

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    d = torch.randn(n_atoms, 3, generator=gen, device=device, dtype=torch.float64)
    d = d / d.norm(dim=1, keepdim=True)
    d[0] = 0
    cur = torch.cumsum(3.8 * d, dim=0)
    out = torch.empty(n_frames, n_atoms, 3, device=device, dtype=torch.float32)
    for f0 in range(0, n_frames, chunk):
        f1 = min(n_frames, f0 + chunk)
        m = f1 - f0
        steps = step_sigma * torch.randn(m, n_atoms, 3, generator=gen, device=device, dtype=torch.float64)
        if f0 == 0:
            steps[0] = 0
        walk = cur.unsqueeze(0) + torch.cumsum(steps, dim=0)
        cur = walk[-1].clone()
        r = _torch_haar(m, gen, device)
        t = trans_sigma * torch.randn(m, 1, 3, generator=gen, device=device, dtype=torch.float64)
        out[f0:f1] = (torch.matmul(walk, r.transpose(1, 2)) + t).to(torch.float32)
    return out
