"""RmsdPlan and PairwiseRmsdPlan with the reference's constructor and run()
signatures (crates/traj-py/src/io.rs:2617-2659 and 2759-2802).

The reference streams FrameChunks of ``chunk_frames`` frames through
``Plan::process_chunk_selected`` (crates/traj-engine/src/executor.rs:471-512)
and, for RmsdPlan, runs rmsd_aligned_selected per frame
(crates/traj-engine/src/plans/rmsd/plan.rs:1161-1248).  Here the whole call is
one C-ABI call: the library streams host frames to the device in chunks and
runs the fused per-frame kernel.  Results are float32 like the reference
(``dtype=np.float64`` gives the unrounded values).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .core import Selection, System, Trajectory
from .dcd import DcdTrajectory

_PAIR_MODES = {"fp32": N.MODE_FP32, "i8x3": N.MODE_I8X3, "i8x2": N.MODE_I8X2, "fp64": N.MODE_FP64}


def parse_device(device: str) -> int:
    """Device::from_spec (crates/traj-engine/src/executor.rs:21-52) restricted
    to CUDA: "auto" and "cuda" mean device 0, "cuda:N" device N."""
    spec = (device or "").strip().lower()
    if spec == "cpu":
        raise N.WarpMdError(N.WMD_ERR_UNSUPPORTED,
                            "unsupported: this warp_md build runs the RMSD plans on CUDA (sm_100a) only")
    if spec in ("auto", "cuda"):
        return 0
    if spec.startswith("cuda"):
        head, _, tail = spec.partition(":")
        if head != "cuda" or not tail or ":" in tail:
            raise RuntimeError(f"parse error: invalid cuda device spec '{device}'")
        try:
            return int(tail)
        except ValueError:
            raise RuntimeError(f"parse error: invalid cuda device spec '{device}'") from None
    raise RuntimeError(f"unsupported: unknown device spec '{device}'")


def parse_reference(value: str) -> str:
    """crates/traj-py/src/pack.rs:2627-2634"""
    if value not in ("topology", "frame0"):
        raise RuntimeError("reference must be 'topology' or 'frame0'")
    return value


def parse_pairwise_metric(value: str) -> str:
    """crates/traj-py/src/pack.rs:2675-2684"""
    if value not in ("rms", "nofit", "dme"):
        raise RuntimeError("metric must be 'rms', 'nofit', or 'dme'")
    return value


def parse_pbc(value: str) -> str:
    if value not in ("none", "orthorhombic"):
        raise RuntimeError("pbc must be 'none' or 'orthorhombic'")
    return value


def frame_subset(n_frames: int, frame_indices: Optional[Sequence[int]]) -> Optional[np.ndarray]:
    """run_plan_with_frame_subset (crates/traj-py/src/pack.rs:1259-1330): when any
    index is negative all are normalised against n_frames
    (executor.rs:210-222), dropping those out of range; otherwise negative-free
    indices are used as given and indices past the end are dropped."""
    if frame_indices is None:
        return None
    raw = [int(i) for i in frame_indices]
    if any(i < 0 for i in raw):
        out = [i + n_frames if i < 0 else i for i in raw]
    else:
        out = raw
    return np.asarray([i for i in out if 0 <= i < n_frames], dtype=np.int64)


def _check_inputs(traj: Trajectory, system: System, selection: Selection) -> np.ndarray:
    if traj.n_atoms() != system.n_atoms():
        raise RuntimeError("mismatch: trajectory atom count does not match system")
    sel = selection.as_array()
    if sel.size and int(sel.max()) >= traj.n_atoms():
        raise RuntimeError("invalid selection: selection index out of range")
    return sel


def _dense_prefix(sel: np.ndarray) -> bool:
    return sel.size == 0 or bool(np.array_equal(sel, np.arange(sel.size, dtype=sel.dtype)))


class RmsdPlan:
    """Per-frame RMSD against a reference (warp_md.RmsdPlan)."""

    def __init__(self, selection: Selection, reference: str = "topology", align: bool = True):
        self.selection = selection
        self.reference_mode = parse_reference(reference)
        self.align = bool(align)

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None, dtype=np.float32) -> np.ndarray:
        dev = parse_device(device)
        sel = _check_inputs(traj, system, self.selection)
        if isinstance(traj, DcdTrajectory) and frame_indices is None:
            return self._run_dcd(traj, system, sel, dtype)
        coords = traj.coords
        sub = frame_subset(coords.shape[0], frame_indices)
        if sub is not None:
            coords = np.ascontiguousarray(coords[sub])
        n_frames = coords.shape[0]
        # reference structure: topology positions0 (plan.rs:188-199) or the
        # first processed frame (plan.rs:336-342)
        if self.reference_mode == "topology":
            if system.positions0 is None:
                raise RuntimeError("mismatch: no topology reference coords")
            ref = system.positions0[sel]
        else:
            if n_frames == 0:
                return np.empty(0, dtype=dtype)
            ref = coords[0][sel]
        if n_frames == 0:
            return np.empty(0, dtype=dtype)
        ctx = N.context(dev)
        r = N.Reference.from_numpy(ctx, ref)
        try:
            out = np.empty(n_frames, np.float64)
            dense = _dense_prefix(sel)
            sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
            ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, coords.ctypes.data, n_frames, coords.shape[1], 3,
                                              N.ptr(sel_arr), int(sel.size), r.handle, int(self.align),
                                              out.ctypes.data, None))
        finally:
            r.close()
        return out.astype(dtype, copy=False)

    def _run_dcd(self, traj: DcdTrajectory, system: System, sel: np.ndarray, dtype) -> np.ndarray:
        """Frames from the trajectory's position to the end of the file, read,
        copied and decoded in batches that overlap the RMSD kernels
        (wmd_dcd_rmsd); the position moves to the end, as the reference's
        streaming run leaves its reader."""
        first = traj._cursor
        n = max(0, traj.n_frames() - first)
        dense = _dense_prefix(sel) and sel.size == traj.n_atoms()
        atoms = None if dense else sel
        if self.reference_mode == "topology":
            if system.positions0 is None:
                raise RuntimeError("mismatch: no topology reference coords")
            ref = system.positions0[sel]
        else:
            if n == 0:
                return np.empty(0, dtype=dtype)
            chunk = traj._read(first, 1, atoms, False)[0]
            ref = chunk[0]
        if sel.size == 0:
            traj._cursor = first + n
            return np.zeros(n, dtype=dtype)
        out = traj.rmsd(ref, atom_indices=atoms, align=self.align, first=first, n=n)
        traj._cursor = first + out.shape[0]
        return out.astype(dtype, copy=False)


def _dme_boxes(traj: Trajectory, n_frames: int, sub: Optional[np.ndarray]) -> np.ndarray:
    """Per-frame orthorhombic box lengths (n_frames, 3) float32 for metric
    "dme" with pbc "orthorhombic".  The trajectory's box is (3,) for every
    frame or (frames, 3), as Trajectory.from_numpy takes it (io.rs:2062-2112);
    without one the reference stops with box_lengths' mismatch
    (crates/traj-core/src/pbc_math.rs:11-15)."""
    b = getattr(traj, "box", None)
    if b is None:
        raise N.WarpMdError(N.WMD_ERR_MISMATCH, "mismatch: orthorhombic box required for PBC")
    a = np.asarray(b, dtype=np.float32)
    if a.ndim == 1:
        if a.shape[0] != 3:
            raise RuntimeError("box must have length 3")
        return np.ascontiguousarray(np.broadcast_to(a, (n_frames, 3)))
    if a.ndim != 2 or a.shape[1] != 3:
        raise RuntimeError("box must have shape (3,) or (frames, 3)")
    if sub is not None:
        a = a[sub]
    if a.shape[0] != n_frames:
        raise RuntimeError("box must have shape (frames, 3)")
    return np.ascontiguousarray(a)


class PairwiseRmsdPlan:
    """All-pairs frame x frame RMSD matrix (warp_md.PairwiseRmsdPlan).

    ``mode`` picks the covariance arithmetic: "i8x3" (tensor cores on
    24-bit fixed-point coordinates split into three int8 limbs, exact integer
    accumulation), "i8x2" (16-bit fixed point), "fp32" (plain FP32 CUDA-core
    tiles) or "fp64" (default; FP64 CUDA-core tiles).  All use an FP64 QCP epilogue."""

    def __init__(self, selection: Selection, metric: str = "rms", pbc: str = "none", mode: str = "fp64"):
        self.selection = selection
        self.metric = parse_pairwise_metric(metric)
        self.pbc = parse_pbc(pbc)
        if mode not in _PAIR_MODES:
            raise RuntimeError(f"mode must be one of {sorted(_PAIR_MODES)}")
        self.mode = mode

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        dev = parse_device(device)
        sel = _check_inputs(traj, system, self.selection)
        coords = traj.coords
        sub = frame_subset(coords.shape[0], frame_indices)
        if sub is not None:
            coords = np.ascontiguousarray(coords[sub])
        n = coords.shape[0]
        out = np.zeros((n, n), np.float32)
        if n == 0:
            return np.zeros((0, 0), np.float32)
        box = _dme_boxes(traj, n, sub) if self.metric == "dme" and self.pbc == "orthorhombic" else None
        ctx = N.context(dev)
        dense = _dense_prefix(sel)
        sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
        if self.metric == "dme":
            ctx.check(ctx.lib.wmd_pairwise_dme(ctx.handle, coords.ctypes.data, n, coords.shape[1], 3, N.ptr(sel_arr),
                                               int(sel.size), N.ptr(box), out.ctypes.data, None))
            return out
        metric = N.PAIR_RMS if self.metric == "rms" else N.PAIR_NOFIT
        ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, coords.ctypes.data, n, coords.shape[1], 3, N.ptr(sel_arr),
                                            int(sel.size), metric, _PAIR_MODES[self.mode], out.ctypes.data, None))
        return out


# ---------------------------------------------------------------------------
# superposition plans
# ---------------------------------------------------------------------------

def _superpose_inputs(plan, traj: Trajectory, system: System, frame_indices):
    """Selection, (subset) frames and reference of a superposition plan: the
    topology positions0 or the first processed frame (plan_exec.rs:82-100,
    131-140), with the selected atoms' masses as weights when mass=True."""
    sel = _check_inputs(traj, system, plan.selection)
    coords = traj.coords
    sub = frame_subset(coords.shape[0], frame_indices)
    if sub is not None:
        coords = np.ascontiguousarray(coords[sub])
    if plan.reference_mode == "topology":
        if system.positions0 is None:
            raise RuntimeError("mismatch: no topology reference coords")
        ref = system.positions0[sel]
    else:
        ref = coords[0][sel] if coords.shape[0] else None
    weights = np.ascontiguousarray(system.masses[sel], dtype=np.float32) if plan.mass else None
    return sel, coords, sub, ref, weights


def superpose_arrays(coords: np.ndarray, sel: np.ndarray, ref: Optional[np.ndarray], weights: Optional[np.ndarray],
                     norotate: bool, apply: bool, device: str = "auto"):
    """Per-frame transforms [F][12] float32 of frames (F, N, 3) onto ``ref``
    (the selected atoms) and, with ``apply``, every atom moved (F, N, 3)."""
    dev = parse_device(device)
    coords = np.ascontiguousarray(coords, dtype=np.float32)
    n_frames, n_atoms = coords.shape[0], coords.shape[1]
    xf = np.empty((n_frames, 12), np.float32)
    out = np.empty((n_frames, n_atoms, 3), np.float32) if apply else None
    if n_frames == 0:
        return xf, out
    ctx = N.context(dev)
    r = N.Reference.from_numpy(ctx, np.asarray(ref, dtype=np.float32).reshape(-1, 3), weights=weights)
    try:
        dense = _dense_prefix(sel)
        sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
        if apply:
            ctx.check(ctx.lib.wmd_superpose(ctx.handle, coords.ctypes.data, n_frames, n_atoms, 3, N.ptr(sel_arr),
                                            int(sel.size), r.handle, int(norotate), out.ctypes.data,
                                            xf.ctypes.data, None))
        else:
            ctx.check(ctx.lib.wmd_superpose_transforms(ctx.handle, coords.ctypes.data, n_frames, n_atoms, 3,
                                                       N.ptr(sel_arr), int(sel.size), r.handle, int(norotate),
                                                       xf.ctypes.data, None))
    finally:
        r.close()
    return xf, out


def _run_superpose(plan, traj: Trajectory, system: System, device: str, frame_indices, apply: bool):
    parse_device(device)
    sel, coords, sub, ref, weights = _superpose_inputs(plan, traj, system, frame_indices)
    if coords.shape[0] == 0:
        return (np.empty((0, 12), np.float32), np.empty((0, coords.shape[1], 3), np.float32) if apply else None,
                sub)
    xf, out = superpose_arrays(coords, sel, ref, weights, plan.norotate, apply, device)
    return xf, out, sub


class AlignPlan:
    """Per-frame superposition transforms (warp_md.AlignPlan,
    crates/traj-py/src/transform.rs:1802-1837): rows of 12 float32 -- R
    row-major (R maps the frame onto the reference) then t = c_ref - R c_frame
    (plan_exec.rs:224-238)."""

    def __init__(self, selection: Selection, reference: str = "topology", mass: bool = False, norotate: bool = False):
        self.selection = selection
        self.reference_mode = parse_reference(reference)
        self.mass = bool(mass)
        self.norotate = bool(norotate)

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None,
            device: str = "auto") -> np.ndarray:
        xf, _, _ = _run_superpose(self, traj, system, device, None, apply=False)
        return xf


class RotationMatrixPlan:
    """Per-frame rotation matrices, (frames, 9) float32 (warp_md.RotationMatrixPlan,
    crates/traj-py/src/correlation.rs:313-349; align_matrix.rs:16-70: the
    first 9 columns of AlignPlan's rows)."""

    def __init__(self, selection: Selection, reference: str = "topology", mass: bool = False):
        self.selection = selection
        self.reference_mode = parse_reference(reference)
        self.mass = bool(mass)
        self.norotate = False

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        xf, _, _ = _run_superpose(self, traj, system, device, frame_indices, apply=False)
        return np.ascontiguousarray(xf[:, :9])


class SuperposePlan:
    """Every atom of every (selected) frame superposed onto the reference
    (warp_md.SuperposePlan, correlation.rs:269-304): a flat float32 series of
    frames x atoms x 3 (plan_exec.rs:431-462)."""

    def __init__(self, selection: Selection, reference: str = "topology", mass: bool = False, norotate: bool = False):
        self.selection = selection
        self.reference_mode = parse_reference(reference)
        self.mass = bool(mass)
        self.norotate = bool(norotate)

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        _, out, _ = _run_superpose(self, traj, system, device, frame_indices, apply=True)
        return out.reshape(-1)


class SuperposeTrajectoryPlan:
    """SuperposePlan returning a trajectory payload (warp_md.SuperposeTrajectoryPlan,
    transform.rs:1839-1875, trajectory_output_to_py transform.rs:1353-1391):
    {"coords": (frames, atoms, 3) float32, "box": (frames, 3) or None,
    "time_ps": (frames,) or None}."""

    def __init__(self, selection: Selection, reference: str = "topology", mass: bool = False, norotate: bool = False):
        self.inner = SuperposePlan(selection, reference, mass, norotate)

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> dict:
        _, out, sub = _run_superpose(self.inner, traj, system, device, frame_indices, apply=True)
        n = out.shape[0]

        def per_frame(values):
            if values is None:
                return None
            a = np.asarray(values)
            if sub is not None and a.shape[0] == traj.coords.shape[0]:
                a = a[sub]
            return a if a.shape[0] == n and n > 0 else None

        box = per_frame(traj.box)
        time = per_frame(traj.time_ps)
        return {"coords": out,
                "box": None if box is None else np.asarray(box, dtype=np.float32).reshape(n, -1)[:, :3],
                "time_ps": None if time is None else np.asarray(time, dtype=np.float32).reshape(n)}


# ---------------------------------------------------------------------------
# fluctuations and per-residue RMSD
# ---------------------------------------------------------------------------

def _fluct_run(plan, traj: Trajectory, system: System, device: str, frame_indices, want_adp: bool):
    dev = parse_device(device)
    sel = _check_inputs(traj, system, plan.selection)
    coords = traj.coords
    sub = frame_subset(coords.shape[0], frame_indices)
    if sub is not None:
        coords = np.ascontiguousarray(coords[sub])
    n_sel = int(sel.size)
    rmsf = np.zeros(n_sel, np.float32)
    adp = np.zeros((n_sel, 6), np.float32) if want_adp else None
    if n_sel == 0 or coords.shape[0] == 0:
        return rmsf, (np.empty((0, 6), np.float32) if want_adp else None)
    ctx = N.context(dev)
    dense = _dense_prefix(sel)
    sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
    ctx.check(ctx.lib.wmd_rmsf(ctx.handle, coords.ctypes.data, coords.shape[0], coords.shape[1], 3, N.ptr(sel_arr),
                               n_sel, rmsf.ctypes.data, None if adp is None else adp.ctypes.data, None))
    return rmsf, adp


class RmsfPlan:
    """Per-atom root-mean-square fluctuation over frames, float32 [n_sel]
    (warp_md.RmsfPlan, crates/traj-py/src/geometry.rs; rms.rs:17-218).  No
    superposition: align the trajectory first (SuperposePlan) when needed."""

    def __init__(self, selection: Selection):
        self.selection = selection

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        return _fluct_run(self, traj, system, device, frame_indices, False)[0]


class AtomicFluctPlan(RmsfPlan):
    """RMSF under its AtomicFluct name (rms.rs:268-300)."""


class BfactorsPlan(RmsfPlan):
    """Pseudo B-factors 8 pi^2 / 3 * rmsf^2 (rms.rs:221-265), float32 [n_sel]."""

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        r = super().run(traj, system, chunk_frames, device, frame_indices).astype(np.float64)
        return (8.0 * np.pi * np.pi / 3.0 * r * r).astype(np.float32)


class AtomicAdpPlan:
    """Per-atom displacement tensors (uxx, uyy, uzz, uxy, uxz, uyz), float32
    [n_sel, 6] (rms.rs:303-429); no rows when there are no frames."""

    def __init__(self, selection: Selection):
        self.selection = selection

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> np.ndarray:
        return _fluct_run(self, traj, system, device, frame_indices, True)[1]


class RmsdPerResPlan:
    """Per-frame, per-residue RMSD after superposing the selection onto the
    reference (warp_md.RmsdPerResPlan, rms.rs:431-686).  run() returns
    (resids int32 [n_res], float32 [frames, n_res]); residues are the
    selection's resids in ascending order, each with its atoms in selection
    order."""

    def __init__(self, selection: Selection, reference: str = "topology", align: bool = True):
        self.selection = selection
        self.reference_mode = parse_reference(reference)
        self.align = bool(align)

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto"):
        dev = parse_device(device)
        sel = _check_inputs(traj, system, self.selection)
        coords = traj.coords
        resids = system.resids[sel] if sel.size else np.zeros(0, np.int64)
        order = np.unique(resids)
        groups = [sel[resids == r] for r in order]
        n_groups = len(groups)
        out = np.zeros((coords.shape[0], n_groups), np.float32)
        resid_arr = order.astype(np.int32)
        if self.reference_mode == "topology":
            if system.positions0 is None:
                raise RuntimeError("mismatch: no topology reference coords")
            ref_all = system.positions0
        else:
            if coords.shape[0] == 0:
                return resid_arr, out
            ref_all = coords[0]
        if coords.shape[0] == 0 or n_groups == 0:
            return resid_arr, out
        ref_all = np.ascontiguousarray(ref_all, dtype=np.float32)
        goff = np.zeros(n_groups + 1, np.uint32)
        goff[1:] = np.cumsum([g.size for g in groups])
        gat = np.ascontiguousarray(np.concatenate(groups), dtype=np.uint32)
        ctx = N.context(dev)
        r = N.Reference.from_numpy(ctx, ref_all[sel])
        groups_ref = N.GroupRef(ctx, ref_all, goff, gat)
        try:
            dense = _dense_prefix(sel)
            sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
            ctx.check(ctx.lib.wmd_rmsd_per_group(ctx.handle, coords.ctypes.data, coords.shape[0], coords.shape[1], 3,
                                                 N.ptr(sel_arr), int(sel.size), r.handle, groups_ref.handle,
                                                 int(self.align), out.ctypes.data, None))
        finally:
            groups_ref.close()
            r.close()
        return resid_arr, out


# ---------------------------------------------------------------------------
# clustering
# ---------------------------------------------------------------------------

class TrajectoryClusterPlan:
    """Frame clustering (warp_md.TrajectoryClusterPlan, crates/traj-py/src/io.rs:
    2805-2881; clustering.rs): DBSCAN over the all-pairs RMSD matrix (computed
    on the tensor-core or SIMT pairwise path, ``pairwise_mode``; "fp64"
    reproduces the reference's matrix) or k-means on frames superposed onto
    frame 0.  run() returns {"labels", "centroids", "sizes", "method",
    "n_frames"}."""

    def __init__(self, selection: Selection, method: str = "dbscan", eps: float = 2.0, min_samples: int = 5,
                 n_clusters: int = 8, max_iter: int = 100, tol: float = 1.0e-4, seed: int = 0,
                 memory_budget_bytes: Optional[int] = None, pairwise_mode: str = "fp64"):
        m = str(method).strip().lower()
        if m not in ("dbscan", "kmeans"):
            raise RuntimeError("method must be 'dbscan' or 'kmeans'")
        if pairwise_mode not in _PAIR_MODES:
            raise RuntimeError(f"pairwise_mode must be one of {sorted(_PAIR_MODES)}")
        self.selection = selection
        self.method = m
        self.eps = float(np.float32(eps))
        self.min_samples = int(min_samples)
        self.n_clusters = int(n_clusters)
        self.max_iter = int(max_iter)
        self.tol = float(np.float32(tol))
        self.seed = int(seed)
        self.memory_budget_bytes = memory_budget_bytes
        self.pairwise_mode = pairwise_mode

    def run(self, traj: Trajectory, system: System, chunk_frames: Optional[int] = None, device: str = "auto",
            frame_indices: Optional[Sequence[int]] = None) -> dict:
        dev = parse_device(device)
        if len(self.selection) == 0:
            raise RuntimeError("mismatch: trajectory_cluster requires a non-empty selection")
        sel = _check_inputs(traj, system, self.selection)
        coords = traj.coords
        sub = frame_subset(coords.shape[0], frame_indices)
        if sub is not None:
            coords = np.ascontiguousarray(coords[sub])
        n = coords.shape[0]
        empty = {"labels": np.zeros(0, np.int32), "centroids": np.zeros(0, np.uint32),
                 "sizes": np.zeros(0, np.uint32), "method": self.method, "n_frames": 0}
        if n == 0:
            return empty
        labels = np.empty(n, np.int32)
        cent = np.empty(n, np.uint32)
        sizes = np.empty(n, np.uint32)
        k = ctypes.c_int64(0)
        ctx = N.context(dev)
        dense = _dense_prefix(sel)
        sel_arr = None if dense else np.ascontiguousarray(sel, dtype=np.uint32)
        if self.method == "dbscan":
            if self.eps <= 0.0:
                raise RuntimeError("parse error: trajectory_cluster DBSCAN eps must be > 0")
            need = n * (n - 1) // 2 * 4
            if self.memory_budget_bytes is not None and need > self.memory_budget_bytes:
                raise RuntimeError(f"unsupported: trajectory_cluster distance matrix requires {need} bytes but "
                                   f"memory_budget_bytes={self.memory_budget_bytes}")
            ctx.check(ctx.lib.wmd_cluster_dbscan(ctx.handle, coords.ctypes.data, n, coords.shape[1], 3, N.ptr(sel_arr),
                                                 int(sel.size), _PAIR_MODES[self.pairwise_mode], self.eps,
                                                 max(1, self.min_samples), labels.ctypes.data, cent.ctypes.data,
                                                 sizes.ctypes.data, k, None))
        else:
            ctx.check(ctx.lib.wmd_cluster_kmeans(ctx.handle, coords.ctypes.data, n, coords.shape[1], 3, N.ptr(sel_arr),
                                                 int(sel.size), self.n_clusters, self.max_iter, self.tol,
                                                 self.seed & 0xFFFFFFFFFFFFFFFF, labels.ctypes.data, cent.ctypes.data,
                                                 sizes.ctypes.data, k, None))
        kk = int(k.value)
        return {"labels": labels, "centroids": cent[:kk].copy(), "sizes": sizes[:kk].copy(), "method": self.method,
                "n_frames": n}
