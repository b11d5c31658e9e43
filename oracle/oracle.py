"""ctypes wrapper over the CPU FP64 oracle (``oracle/rmsd_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / ``--impl reference`` legs of ``bench.py``, always as the
checker.  The product (``warp-md_b200/warp_md``) never imports it.

The C file restates warp-md's RMSD plans (see its header for the file:line
citations into crates/traj-engine/src/plans/rmsd/plan.rs).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librmsd_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int
_vp = ctypes.c_void_p


def build() -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.wmdo_rmsd_frames.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _vp, _int, _int, _vp, _vp, _int]
        L.wmdo_rmsd_frames.restype = None
        L.wmdo_rmsd_grad.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _vp, _int, _vp, _vp, _int]
        L.wmdo_rmsd_grad.restype = None
        L.wmdo_pairwise_block.argtypes = [_vp, _i64, _i64, _int, _int, _i64, _i64, _i64, _i64, _vp, _vp, _i64, _int]
        L.wmdo_pairwise_block.restype = None
        L.wmdo_pairwise_dme.argtypes = [_vp, _i64, _i64, _int, _vp, _vp, _vp, _int]
        L.wmdo_pairwise_dme.restype = None
        L.wmdo_qcp_rmsd.argtypes = [_vp, _vp, _i64, _int, _int]
        L.wmdo_qcp_rmsd.restype = ctypes.c_double
        L.wmdo_svd3.argtypes = [_f64p, _f64p, _f64p, _f64p]
        L.wmdo_svd3.restype = _int
        L.wmdo_kabsch_rotation.argtypes = [_f64p, _f64p, ctypes.POINTER(ctypes.c_double)]
        L.wmdo_kabsch_rotation.restype = None
        L.wmdo_superpose.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _vp, _int, _vp, _int, _vp, _vp, _int]
        L.wmdo_superpose.restype = None
        L.wmdo_rmsf.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _vp, _vp]
        L.wmdo_rmsf.restype = None
        L.wmdo_rmsd_perres.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _vp, _vp, _vp, _i64, _int, _vp]
        L.wmdo_rmsd_perres.restype = None
        L.wmdo_dbscan.argtypes = [_vp, _i64, ctypes.c_double, _i64, _vp, _vp, _vp]
        L.wmdo_dbscan.restype = _i64
        L.wmdo_kmeans.argtypes = [_vp, _i64, _i64, _int, _vp, _i64, _i64, _i64, ctypes.c_double, ctypes.c_uint64, _vp,
                                  _vp, _vp]
        L.wmdo_kmeans.restype = _i64
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _coords(coords) -> Tuple[np.ndarray, int]:
    c = np.ascontiguousarray(coords, dtype=np.float32)
    if c.ndim == 2:
        c = c[None]
    if c.ndim != 3 or c.shape[2] not in (3, 4):
        raise ValueError("coords must be (frames, atoms, 3|4)")
    return c, c.shape[2]


def rmsd_frames(coords, reference, selection=None, align: bool = True, threads: int = 0):
    """RmsdPlan semantics: reference holds the selected atoms (n_sel, 3|4).
    Returns (f32 array as the reference returns it, f64 array before rounding)."""
    c, stride = _coords(coords)
    ref = np.ascontiguousarray(reference, dtype=np.float32)
    n_sel = ref.shape[0]
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    if sel is not None and sel.shape[0] != n_sel:
        raise ValueError("selection and reference lengths differ")
    out32 = np.empty(c.shape[0], np.float32)
    out64 = np.empty(c.shape[0], np.float64)
    lib().wmdo_rmsd_frames(_ptr(c), c.shape[0], c.shape[1], stride, _ptr(sel), n_sel, _ptr(ref),
                           ref.shape[1], int(bool(align)), _ptr(out32), _ptr(out64), int(threads))
    return out32, out64


def rmsd_grad(coords, reference, selection=None, threads: int = 0):
    """Analytic FP64 gradient dRMSD/dx, shape (frames, atoms, 3); rows of
    unselected atoms are zero.  Returns (rmsd f64, grad f64)."""
    c, stride = _coords(coords)
    ref = np.ascontiguousarray(reference, dtype=np.float32)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    rm = np.empty(c.shape[0], np.float64)
    g = np.zeros((c.shape[0], c.shape[1], 3), np.float64)
    lib().wmdo_rmsd_grad(_ptr(c), c.shape[0], c.shape[1], stride, _ptr(sel), ref.shape[0], _ptr(ref),
                         ref.shape[1], _ptr(rm), _ptr(g), int(threads))
    return rm, g


def pairwise(frames, metric: str = "rms", block=None, threads: int = 0):
    """PairwiseRmsdPlan::finalize semantics over already-selected frames.
    block = (i0, i1, j0, j1) restricts to a sub-block.  Returns (f32, f64)."""
    c, stride = _coords(frames)
    n = c.shape[0]
    i0, i1, j0, j1 = block if block is not None else (0, n, 0, n)
    m = {"rms": 0, "nofit": 1}[metric]
    out32 = np.empty((i1 - i0, j1 - j0), np.float32)
    out64 = np.empty((i1 - i0, j1 - j0), np.float64)
    lib().wmdo_pairwise_block(_ptr(c), n, c.shape[1], stride, m, i0, i1, j0, j1, _ptr(out32), _ptr(out64),
                              j1 - j0, int(threads))
    return out32, out64


def pairwise_dme(frames, box=None, threads: int = 0):
    """PairwiseRmsdPlan metric "dme" over already-selected frames; box =
    per-frame orthorhombic lengths (n_frames, 3) for pbc "orthorhombic", or
    None.  Returns (f32, f64) matrices."""
    c, stride = _coords(frames)
    n = c.shape[0]
    b = None if box is None else np.ascontiguousarray(np.broadcast_to(np.asarray(box, np.float32), (n, 3)))
    out32 = np.empty((n, n), np.float32)
    out64 = np.empty((n, n), np.float64)
    lib().wmdo_pairwise_dme(_ptr(c), n, c.shape[1], stride, _ptr(b), _ptr(out32), _ptr(out64), int(threads))
    return out32, out64


def qcp_rmsd(x, y, high_precision: bool = False) -> float:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    return float(lib().wmdo_qcp_rmsd(_ptr(x), _ptr(y), x.shape[0], x.shape[1], int(high_precision)))


def svd3(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    u = np.empty(9); s = np.empty(3); vt = np.empty(9)
    lib().wmdo_svd3(a, u, s, vt)
    return u.reshape(3, 3), s, vt.reshape(3, 3)


def kabsch_rotation(h):
    h = np.ascontiguousarray(h, dtype=np.float64).reshape(9)
    r = np.empty(9)
    ss = ctypes.c_double()
    lib().wmdo_kabsch_rotation(h, r, ctypes.byref(ss))
    return r.reshape(3, 3), ss.value


def superpose(coords, reference, selection=None, weights=None, norotate: bool = False, apply: bool = True,
              threads: int = 0):
    """AlignPlan / SuperposePlan semantics: per-frame transforms [F][12] (R
    row-major, t; FP64) and, with apply, every atom moved (float32 [F][N][3])."""
    c, stride = _coords(coords)
    ref = np.ascontiguousarray(reference, dtype=np.float32)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    if sel is not None and sel.shape[0] != ref.shape[0]:
        raise ValueError("selection and reference lengths differ")
    xf = np.empty((c.shape[0], 12), np.float64)
    out = np.empty((c.shape[0], c.shape[1], 3), np.float32) if apply else None
    lib().wmdo_superpose(_ptr(c), c.shape[0], c.shape[1], stride, _ptr(sel), ref.shape[0], _ptr(ref), ref.shape[1],
                         _ptr(w), int(bool(norotate)), _ptr(xf), _ptr(out), int(threads))
    return xf, out


def rmsf(coords, selection=None, n_sel=None):
    """RmsfPlan (Welford, FP64) and AtomicAdpPlan moments.  Returns (rmsf [n_sel],
    adp [n_sel][6]) in FP64."""
    c, stride = _coords(coords)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    n = sel.shape[0] if sel is not None else (c.shape[1] if n_sel is None else n_sel)
    r = np.zeros(n, np.float64)
    a = np.zeros((n, 6), np.float64)
    lib().wmdo_rmsf(_ptr(c), c.shape[0], c.shape[1], stride, _ptr(sel), n, _ptr(r), _ptr(a))
    return r, a


def rmsd_perres(coords, ref_all, groups, selection=None, align: bool = True):
    """RmsdPerResPlan CPU path.  groups: list of atom-index lists.  Returns FP64
    [frames][groups]."""
    c, stride = _coords(coords)
    ref = np.ascontiguousarray(ref_all, dtype=np.float32)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    n_sel = sel.shape[0] if sel is not None else c.shape[1]
    goff = np.zeros(len(groups) + 1, np.uint32)
    goff[1:] = np.cumsum([len(g) for g in groups])
    gat = np.ascontiguousarray(np.concatenate([np.asarray(g, np.uint32) for g in groups]) if groups else
                               np.zeros(1, np.uint32), dtype=np.uint32)
    out = np.zeros((c.shape[0], len(groups)), np.float64)
    lib().wmdo_rmsd_perres(_ptr(c), c.shape[0], c.shape[1], stride, _ptr(sel), n_sel, _ptr(ref), _ptr(goff),
                           _ptr(gat), len(groups), int(bool(align)), _ptr(out))
    return out


def dbscan(dist, eps: float, min_samples: int):
    """TrajectoryClusterPlan's DBSCAN over an (n, n) float32 matrix; eps is
    taken as float32 then widened, as the plan stores it.  Returns (labels
    int32, centroids uint32, sizes uint32)."""
    d = np.ascontiguousarray(dist, dtype=np.float32)
    n = d.shape[0]
    labels = np.empty(n, np.int32)
    cent = np.empty(max(n, 1), np.uint32)
    sizes = np.empty(max(n, 1), np.uint32)
    k = lib().wmdo_dbscan(_ptr(d), n, float(np.float32(eps)), int(min_samples), _ptr(labels), _ptr(cent), _ptr(sizes))
    return labels, cent[:k].copy(), sizes[:k].copy()


def kmeans(coords, selection=None, n_clusters=8, max_iter=100, tol=1e-4, seed=0):
    """TrajectoryClusterPlan's k-means.  tol is taken as float32 then widened,
    as the plan stores it.  Returns (labels, centroids, sizes)."""
    c, stride = _coords(coords)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.uint32)
    n_sel = sel.shape[0] if sel is not None else c.shape[1]
    n = c.shape[0]
    labels = np.empty(max(n, 1), np.int32)
    cent = np.empty(max(n, 1), np.uint32)
    sizes = np.empty(max(n, 1), np.uint32)
    k = lib().wmdo_kmeans(_ptr(c), n, c.shape[1], stride, _ptr(sel), n_sel, int(n_clusters), int(max_iter),
                          float(np.float32(tol)), int(seed), _ptr(labels), _ptr(cent), _ptr(sizes))
    return labels[:n].copy(), cent[:k].copy(), sizes[:k].copy()
