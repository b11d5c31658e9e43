"""Per-frame RMSD (+ dRMSD/dx) of many trajectories of uneven size at once.

``BatchedRmsd(coords, refs, with_grad)`` prepares one persistent launch over
all trajectories (``wmd_batched_prepare``: validation, workspace, trajectory
table, tile shape chosen by timing); ``run()`` then only enqueues kernels on
the current stream, and ``graph()`` captures that launch in a CUDA graph.
The values equal ``torch_ops.rmsd`` per trajectory (align on, all atoms);
``grads[i][f]`` is d rmsd_i[f] / d coords_i[f].  The reference has no batched
form: it runs one ``RmsdPlan`` per trajectory (crates/traj-engine/src/plans/
rmsd/plan.rs:164-418).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import torch

from . import _native as N


class BatchedRmsd:
    def __init__(self, coords: Sequence[torch.Tensor], refs: Sequence[torch.Tensor], with_grad: bool = False):
        if len(coords) != len(refs):
            raise N.WarpMdError(N.WMD_ERR_MISMATCH, "coords and refs differ in length")
        if len(coords) == 0:
            raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, "empty batch")
        dev = coords[0].device
        if dev.type != "cuda":
            raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, "coords must be CUDA tensors")
        self.coords: List[torch.Tensor] = []
        self.refs: List[torch.Tensor] = []
        for i, (x, y) in enumerate(zip(coords, refs)):
            if x.device != dev or y.device != dev:
                raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, f"trajectory {i}: all tensors must be on {dev}")
            if x.dtype != torch.float32 or x.dim() != 3 or x.shape[2] != 3:
                raise N.WarpMdError(N.WMD_ERR_INVALID_ARG, f"trajectory {i}: coords must be float32 (frames, atoms, 3)")
            if tuple(y.shape) != (x.shape[1], 3):
                raise N.WarpMdError(N.WMD_ERR_MISMATCH, f"trajectory {i}: reference shape {tuple(y.shape)} "
                                                        f"!= ({x.shape[1]}, 3)")
            x = x.contiguous()
            if x.data_ptr() % 16:
                x = x.clone()
            self.coords.append(x)
            self.refs.append(y.to(torch.float32).contiguous())
        self.device = dev
        self.with_grad = bool(with_grad)
        self.rmsd = [torch.zeros(x.shape[0], dtype=torch.float64, device=dev) for x in self.coords]
        self.grads: Optional[List[torch.Tensor]] = (
            [torch.zeros_like(x) for x in self.coords] if self.with_grad else None)
        self.ctx = N.Context(dev.index or 0)  # one context per batch: it holds the prepared launch
        n = len(self.coords)
        self._descs = (N.BatchDesc * n)()
        for i, x in enumerate(self.coords):
            d = self._descs[i]
            d.coords = x.data_ptr() if x.numel() else None
            d.ref = self.refs[i].data_ptr() if self.refs[i].numel() else None
            d.n_atoms = x.shape[1]
            d.n_frames = x.shape[0]
            d.rmsd = self.rmsd[i].data_ptr() if x.shape[0] else None
            d.grad = self.grads[i].data_ptr() if (self.with_grad and x.numel()) else None
        self._n = n
        with torch.cuda.device(dev):
            torch.cuda.current_stream().synchronize()
            self.ctx.check(self.ctx.lib.wmd_batched_prepare(self.ctx.handle, self._descs, n, int(self.with_grad)))

    def run(self, stream: Optional[torch.cuda.Stream] = None) -> List[torch.Tensor]:
        """Enqueues the batch on ``stream`` (default: the current stream);
        returns the per-trajectory RMSD tensors (float64), written in place."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.ctx.check(self.ctx.lib.wmd_batched_rmsd(self.ctx.handle, self._descs, self._n, int(self.with_grad),
                                                     s.cuda_stream))
        return self.rmsd

    def graph(self) -> torch.cuda.CUDAGraph:
        """Captures one ``run()`` in a CUDA graph (replay re-reads the same
        coordinate buffers, so update them in place between replays)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run(s)  # warm launch outside capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        with torch.cuda.graph(g, stream=s):
            self.run(s)
        return g

    def layout(self) -> dict:
        """The layout the prepare step's autotuner chose."""
        t, fm = ctypes.c_int(), ctypes.c_int()
        self.ctx.check(self.ctx.lib.wmd_batched_layout(self.ctx.handle, ctypes.byref(t), ctypes.byref(fm)))
        return {"tile_atoms": t.value, "frame_major": fm.value == 1,
                "layout": {0: "tiles", 1: "frames", 2: "lanes"}.get(fm.value, str(fm.value))}

    def close(self) -> None:
        self.ctx.close()
