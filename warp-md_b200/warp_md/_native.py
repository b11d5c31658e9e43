"""ctypes binding of libwarpmd_rmsd.so (the C ABI in include/warpmd_rmsd.h).

The library is built in-tree by ``warp-md_b200/build_native.py`` into
``warp_md/_native/``.  There is no CPU implementation behind this module: when
the library or a CUDA device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Dict, Optional

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_native", "libwarpmd_rmsd.so")

WMD_OK = 0
WMD_ERR_INVALID_ARG = -1
WMD_ERR_CUDA = -2
WMD_ERR_OOM = -3
WMD_ERR_MISMATCH = -4
WMD_ERR_UNSUPPORTED = -5
WMD_ERR_TIMEOUT = -6
WMD_ERR_NO_DEVICE = -7
WMD_ERR_IO = -8
WMD_ERR_PARSE = -9

PAIR_RMS = 0
PAIR_NOFIT = 1
PAIR_DME = 2

MODE_FP32 = 0
MODE_I8X3 = 1
MODE_I8X2 = 2
MODE_FP64 = 3

FRAME_STATS = 16

# every symbol include/warpmd_rmsd.h declares
EXPORTED = (
    "wmd_create", "wmd_destroy", "wmd_last_error", "wmd_version", "wmd_reference_upload", "wmd_reference_free",
    "wmd_rmsd_frames", "wmd_rmsd_forward", "wmd_rmsd_backward", "wmd_rmsd_covariance", "wmd_pairwise_rmsd", "wmd_pairwise_dme",
    "wmd_batched_prepare", "wmd_batched_rmsd", "wmd_batched_layout", "wmd_rmsd_frames_noalloc", "wmd_set_wait_test",
    "wmd_pairwise_rmsd_part", "wmd_rmsd_backward_f64", "wmd_rmsd_value_and_grad",
    "wmd_reference_upload_weighted", "wmd_superpose_transforms", "wmd_superpose", "wmd_rmsf", "wmd_rmsd_per_group",
    "wmd_group_ref_upload", "wmd_group_ref_free", "wmd_cluster_dbscan", "wmd_cluster_kmeans", "wmd_dcd_open",
    "wmd_dcd_close", "wmd_dcd_info", "wmd_dcd_read", "wmd_dcd_rmsd",
)


class WarpMdError(RuntimeError):
    """Raised for every failing library call (the reference raises RuntimeError
    for TrajError values, crates/traj-py/src/pack.rs:1188-1190)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class BatchDesc(ctypes.Structure):
    _fields_ = [
        ("coords", ctypes.c_void_p),
        ("ref", ctypes.c_void_p),
        ("n_atoms", ctypes.c_int64),
        ("n_frames", ctypes.c_int64),
        ("rmsd", ctypes.c_void_p),
        ("grad", ctypes.c_void_p),
    ]


_lib = None
_lib_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Loads the native library (raises if it has not been built)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise WarpMdError(WMD_ERR_UNSUPPORTED,
                              f"native library missing: {LIB_PATH} (run warp-md_b200/build_native.py)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        L.wmd_create.argtypes = [i32, ctypes.POINTER(vp)]
        L.wmd_destroy.argtypes = [vp]
        L.wmd_last_error.argtypes = [vp]
        L.wmd_last_error.restype = ctypes.c_char_p
        L.wmd_version.argtypes = []
        L.wmd_version.restype = ctypes.c_char_p
        L.wmd_reference_upload.argtypes = [vp, vp, i64, i32, ctypes.POINTER(vp)]
        L.wmd_reference_free.argtypes = [vp, vp]
        L.wmd_set_wait_test.argtypes = [vp, ctypes.c_uint64, i32]
        L.wmd_rmsd_frames.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, i32, vp, vp]
        L.wmd_rmsd_forward.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp, vp]
        L.wmd_rmsd_backward.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp, vp, vp]
        L.wmd_rmsd_backward_f64.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp, i64, vp, vp]
        L.wmd_rmsd_value_and_grad.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, i64, vp, vp, vp]
        L.wmd_rmsd_covariance.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp, vp, vp]
        L.wmd_pairwise_rmsd.argtypes = [vp, vp, i64, i64, i32, vp, i64, i32, i32, vp, vp]
        L.wmd_pairwise_rmsd_part.argtypes = [vp, vp, i64, i64, i32, vp, i64, i32, i32, i32, i32, vp, vp]
        L.wmd_pairwise_dme.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp]
        L.wmd_batched_prepare.argtypes = [vp, ctypes.POINTER(BatchDesc), i32, i32]
        L.wmd_batched_rmsd.argtypes = [vp, ctypes.POINTER(BatchDesc), i32, i32, vp]
        L.wmd_batched_layout.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        L.wmd_reference_upload_weighted.argtypes = [vp, vp, i64, i32, vp, ctypes.POINTER(vp)]
        L.wmd_superpose_transforms.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, i32, vp, vp]
        L.wmd_superpose.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, i32, vp, vp, vp]
        L.wmd_rmsf.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, vp]
        L.wmd_rmsd_per_group.argtypes = [vp, vp, i64, i64, i32, vp, i64, vp, vp, i32, vp, vp]
        L.wmd_group_ref_upload.argtypes = [vp, vp, i64, i32, vp, vp, i64, ctypes.POINTER(vp)]
        L.wmd_group_ref_free.argtypes = [vp, vp]
        L.wmd_cluster_dbscan.argtypes = [vp, vp, i64, i64, i32, vp, i64, i32, ctypes.c_float, i64, vp, vp, vp,
                                         ctypes.POINTER(i64), vp]
        L.wmd_cluster_kmeans.argtypes = [vp, vp, i64, i64, i32, vp, i64, i64, i64, ctypes.c_float, ctypes.c_uint64,
                                         vp, vp, vp, ctypes.POINTER(i64), vp]
        L.wmd_rmsd_frames_noalloc.argtypes = [vp, i64, i64, i32, vp, i64, i32, vp, vp]
        L.wmd_dcd_open.argtypes = [vp, ctypes.c_char_p, ctypes.c_float, ctypes.POINTER(vp)]
        L.wmd_dcd_close.argtypes = [vp, vp]
        L.wmd_dcd_info.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)]
        L.wmd_dcd_read.argtypes = [vp, vp, i64, i64, vp, i64, vp, vp, vp, ctypes.POINTER(i64), vp]
        L.wmd_dcd_rmsd.argtypes = [vp, vp, i64, i64, vp, i64, vp, i32, vp, ctypes.POINTER(i64), vp]
        for name in EXPORTED:
            getattr(L, name).restype = getattr(L, name).restype if name in ("wmd_last_error", "wmd_version") else i32
        _lib = L
        return _lib


def version() -> str:
    return load().wmd_version().decode()


class Context:
    """Owns one wmd_ctx (one CUDA device; not shared between threads)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.wmd_create(int(device), ctypes.byref(h))
        if rc != WMD_OK:
            raise WarpMdError(rc, self.lib.wmd_last_error(None).decode())
        self.handle = h

    def check(self, rc: int) -> None:
        if rc != WMD_OK:
            raise WarpMdError(rc, self.lib.wmd_last_error(self.handle).decode())

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.wmd_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


class Reference:
    """A reference structure uploaded to the device (wmd_ref)."""

    def __init__(self, ctx: Context, coords_ptr: int, n_sel: int, stride: int, keepalive=None, weights_ptr=None):
        self.ctx = ctx
        self.n_sel = int(n_sel)
        h = ctypes.c_void_p()
        if weights_ptr is None:
            ctx.check(ctx.lib.wmd_reference_upload(ctx.handle, coords_ptr, int(n_sel), int(stride), ctypes.byref(h)))
        else:
            ctx.check(ctx.lib.wmd_reference_upload_weighted(ctx.handle, coords_ptr, int(n_sel), int(stride),
                                                            weights_ptr, ctypes.byref(h)))
        self.handle = h
        self._keep = keepalive

    @classmethod
    def from_numpy(cls, ctx: Context, ref: np.ndarray, weights: Optional[np.ndarray] = None) -> "Reference":
        r = np.ascontiguousarray(ref, dtype=np.float32)
        if r.ndim != 2 or r.shape[1] not in (3, 4):
            raise WarpMdError(WMD_ERR_INVALID_ARG, "reference must have shape (atoms, 3) or (atoms, 4)")
        if weights is None:
            return cls(ctx, r.ctypes.data, r.shape[0], r.shape[1], keepalive=r)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        if w.shape != (r.shape[0],):
            raise WarpMdError(WMD_ERR_MISMATCH, "weights must have one entry per reference atom")
        return cls(ctx, r.ctypes.data, r.shape[0], r.shape[1], keepalive=(r, w), weights_ptr=w.ctypes.data)

    def close(self) -> None:
        if getattr(self, "handle", None) and self.ctx.handle:
            self.ctx.lib.wmd_reference_free(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class GroupRef:
    """Atom groups with the all-atom reference (wmd_group_ref)."""

    def __init__(self, ctx: Context, ref_all: np.ndarray, offsets: np.ndarray, atoms: np.ndarray):
        self.ctx = ctx
        r = np.ascontiguousarray(ref_all, dtype=np.float32)
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        at = np.ascontiguousarray(atoms, dtype=np.uint32) if len(atoms) else np.zeros(1, np.uint32)
        self.n_groups = off.size - 1
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wmd_group_ref_upload(ctx.handle, r.ctypes.data, r.shape[0], r.shape[1], off.ctypes.data,
                                               at.ctypes.data, self.n_groups, ctypes.byref(h)))
        self.handle = h

    def close(self) -> None:
        if getattr(self, "handle", None) and self.ctx.handle:
            self.ctx.lib.wmd_group_ref_free(self.ctx.handle, self.handle)
        self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


_contexts: Dict[int, Context] = {}
_ctx_lock = threading.Lock()


def context(device: int = 0) -> Context:
    """Process-wide default context per device (created on first use)."""
    with _ctx_lock:
        ctx = _contexts.get(device)
        if ctx is None:
            ctx = Context(device)
            _contexts[device] = ctx
        return ctx


def ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data
