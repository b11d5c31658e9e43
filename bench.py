"""Benchmark of the RMSD hot path on B200.

Headline: streaming per-frame RMSD + QCP superposition, 100,000-atom selection
x 10,000 frames of float32 coordinates (12 GB resident), reported as
atom-frames/s.  One step = one pass of the per-frame kernel over all frames.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: device-resident frames, K steps timed with CUDA events on the
  launching stream between barrier + synchronize, max over ranks; inputs (12
  GB per GPU) are far larger than L2, so no flush is needed.
* e2e: the same metric through the C ABI with pinned HOST buffers -- every step
  copies the step's frames host->device inside the call and reads the RMSD
  vector back.
* roofline: algorithmic bytes = 12 B per atom-frame (coordinates read once) +
  8 B per frame (result), over the kernel's event-timed duration, against the
  measured HBM copy bandwidth.
* cpu_baseline: the C FP64 restatement of the reference's CPU path
  (oracle/, rmsd_aligned_selected) on a bounded sample of the same workload.
* pairwise: the 20,000-frame x 1,000-atom all-pairs matrix, plain FP32 form
  vs the tensor-core forms, errors against the FP64 oracle on 512 x 512.
* differentiable: 4,096 frames x 2,000 atoms, forward + backward through
  torch.autograd (L2 flushed before each step).
* batched_uneven: 512 trajectories (atoms log-uniform 50-20,000, frames
  uniform 100-5,000), forward + gradients, one graph-replayed batched launch
  vs one forward + backward call per trajectory.
* superpose: 100,000-atom frames x 2,000 frames, mass-weighted 10,000-atom
  selection, transforms + every atom moved (SuperposePlan).
* fluct: RMSF + ADP over 100,000 atoms x 2,000 frames, and per-residue RMSD
  of 10,000 residues after superposing a 10,000-atom selection.
* cluster: DBSCAN over the 20,000-frame all-pairs matrix (tensor-core and
  FP64 forms) and k-means on the superposed frames (TrajectoryClusterPlan).
* --gpus N (torchrun): weak scaling, each rank streams its own 10,000 frames;
  no data-path collective (frames are independent).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "warp-md_b200"))

N_ATOMS = 100_000
N_FRAMES = 10_000
SIGMA = (0.05, 3.0)
BYTES_PER_UNIT = 12.0        # float32 xyz read once per atom-frame
BYTES_PER_FRAME_OUT = 8.0    # one float64 per frame
METRIC = "RMSD atom-frames/s"
UNIT = "atom-frames/s"
WORKLOAD = ("streaming per-frame RMSD+QCP superposition: 100,000-atom selection x 10,000 frames, float32 xyz "
            "(12 GB resident), random-walk reference, Haar rotations, N(0,10 A) translations, "
            "sigma ~ U(0.05, 3.0) A per frame")


def _measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(threads: int, n_frames: int, seed: int = 7, frames=None, ref=None):
    """Times the oracle (C FP64 restatement of the reference CPU path,
    rmsd_aligned_selected) on a bounded sample of the streaming workload:
    the given host frames, or freshly generated ones."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle
    from warp_md import synth

    if frames is None:
        frames, ref = synth.make_trajectory(N_ATOMS, n_frames, SIGMA, seed=seed)
    fr = frames[:n_frames]
    oracle.rmsd_frames(fr[:2], ref, threads=threads)  # warm
    t0 = time.perf_counter()
    _, vals = oracle.rmsd_frames(fr, ref, threads=threads)
    dt = time.perf_counter() - t0
    return (N_ATOMS * fr.shape[0]) / dt, dt, vals


PAIR_ATOMS = 1000
PAIR_WORKLOAD = ("all-pairs 2D-RMSD matrix: 20,000 frames x 1,000 atoms, slow random drift (N(0, 0.1 A) per "
                 "atom per frame) under per-frame random rigid motions, float32")


def _bf16_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def run_pairwise(args, ctx, stream, rank):
    """All-pairs workload: plain FP32 CUDA-core form vs the tensor-core forms
    (int8 limbs, exact int32 accumulation), each with an FP64 QCP epilogue.
    Errors are measured against the FP64 oracle on a 512 x 512 block."""
    import numpy as np
    import torch

    from warp_md import _native as N
    from warp_md import synth
    from warp_md.plans import _PAIR_MODES

    F = args.pair_frames
    n = PAIR_ATOMS
    coords = synth.make_drift_trajectory_torch(n, F, 0.1, seed=3 + rank, device="cuda")
    out = torch.empty(F, F, dtype=torch.float32, device="cuda")
    pairs = F * (F - 1) / 2
    res = {"metric": "2D-RMSD pairs/s", "unit": "pairs/s", "config": PAIR_WORKLOAD, "n_frames": F, "n_atoms": n}
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    blk = min(512, F)
    host_blk = coords[:blk].cpu().numpy()
    _, exact = oracle.pairwise(host_blk, "rms")
    peak, peak_kind = _bf16_peak()
    n_pad64 = (n + 63) // 64 * 64
    for mode in args.pair_modes.split(","):
        def step():
            ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, coords.data_ptr(), F, n, 3, None, n, N.PAIR_RMS,
                                                _PAIR_MODES[mode], out.data_ptr(), stream.cuda_stream))
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.pair_steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.pair_steps
        got = out[:blk, :blk].cpu().numpy()
        err = np.abs(got - exact)
        entry = {"ms": ms, "value": pairs / (ms / 1e3), "max_err_A": float(err.max()),
                 "rms_err_A": float(np.sqrt((err ** 2).mean())),
                 "useful_tflops": 18.0 * n * pairs / (ms / 1e3) / 1e12}
        if mode in ("i8x3", "i8x2"):
            limbs = 3 if mode == "i8x3" else 2
            ni, nj = (F + 39) // 40, (F + 29) // 30
            tiles = sum(1 for bi in range(ni) for bj in range(nj)
                        if bi * 40 < min((bj + 1) * 30, F) - 1)
            issued = 2.0 * 128 * 96 * limbs * limbs * n_pad64 * tiles
            ach = issued / (ms / 1e3) / 1e12
            entry["roofline"] = {"bound": "tensor", "achieved": ach, "peak": 2 * peak, "unit": "TOP/s (int8)",
                                 "frac": ach / (2 * peak),
                                 "peak_source": f"2 x {peak_kind} dense bf16 ({peak} TFLOP/s, MEASURED_PEAKS.json): "
                                                "int8 MMA rate is twice the bf16 rate",
                                 "issued_int8_ops": issued, "note": "includes whole tile launches"}
        res[mode] = entry
    if "fp32" in res and "i8x3" in res:
        res["speedup_i8x3_vs_fp32"] = res["fp32"]["ms"] / res["i8x3"]["ms"]
    if "fp32" in res and "i8x2" in res:
        res["speedup_i8x2_vs_fp32"] = res["fp32"]["ms"] / res["i8x2"]["ms"]
    del out, coords
    torch.cuda.empty_cache()
    return res


def _l2_flush_buffer():
    import torch

    return torch.empty(256 << 20, dtype=torch.uint8, device="cuda")


def run_differentiable(args, stream, rank):
    """Differentiable RMSD: 4,096 frames x 2,000 atoms (98 MB, smaller than
    L2), forward + hand-written backward.  Three forms of the step, each timed
    with L2 flushed (256 MB write) before it: torch.autograd eagerly, the same
    autograd step replayed from a CUDA graph, and rmsd_value_and_grad (value
    and gradient in one launch).  Algorithmic bytes: x read once and the
    gradient written once, 24 B per atom-frame, + 8 B per frame."""
    import numpy as np
    import torch

    from warp_md import synth
    from warp_md.torch_ops import rmsd, rmsd_value_and_grad

    F, n = 4096, 2000
    x, ref = synth.make_trajectory_torch(n, F, 0.3, seed=17 + rank, device="cuda")
    x.requires_grad_(True)
    flush = _l2_flush_buffer()

    def step():
        x.grad = None
        v = rmsd(x, ref)
        v.sum().backward()
        return v

    def timed(fn, reps):
        times = []
        for _ in range(reps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        return statistics.median(times)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ms_eager = timed(step, args.diff_steps)
    g_autograd = x.grad.detach().clone()

    # the same autograd step captured once and replayed
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            step()
    torch.cuda.current_stream().wait_stream(side)
    x.grad = None
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        v = rmsd(x, ref)
        v.sum().backward()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    ms_graph = timed(graph.replay, args.diff_steps)
    graph_diff = float((x.grad - g_autograd).abs().max().item())

    xd = x.detach()
    for _ in range(3):
        rmsd_value_and_grad(xd, ref)
    torch.cuda.synchronize()
    ms_vg_call = timed(lambda: rmsd_value_and_grad(xd, ref), args.diff_steps)
    # the same call into preallocated outputs, replayed from a CUDA graph
    val_vg = torch.empty(F, dtype=torch.float64, device="cuda")
    g_vg = torch.empty_like(xd)
    rmsd_value_and_grad(xd, ref, out=val_vg, grad=g_vg)
    torch.cuda.synchronize()
    vg_graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(vg_graph):
        rmsd_value_and_grad(xd, ref, out=val_vg, grad=g_vg)
    for _ in range(3):
        vg_graph.replay()
    torch.cuda.synchronize()
    ms_vg = timed(vg_graph.replay, args.diff_steps)
    vg_diff = float((g_vg - g_autograd).abs().max().item())
    # oracle check on 16 frames: RMSD and analytic FP64 gradient
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    idx = torch.arange(0, F, F // 16, device="cuda")
    rm, go = oracle.rmsd_grad(xd.index_select(0, idx).cpu().numpy(), ref.cpu().numpy())
    rerr = float(np.abs(val_vg.index_select(0, idx).cpu().numpy() - rm).max())
    gerr = float(np.abs(g_vg.index_select(0, idx).cpu().numpy() - go).max() / np.abs(go).max())
    ok = bool(torch.isfinite(g_vg).all().item())
    del graph, vg_graph, v, x, g_vg, g_autograd, xd, flush
    torch.cuda.empty_cache()
    peak, _ = _measured_peaks()
    alg = 24.0 * n * F + 8.0 * F

    def entry(ms, how):
        return {"ms": ms, "value": n * F / (ms / 1e3), "how": how,
                "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg / (ms / 1e3) / 1e9 / peak, "bytes_per_atom_frame": 24}}

    eager = entry(ms_eager, "torch.autograd: rmsd(x, ref).sum().backward(), eager")
    graphed = entry(ms_graph, "the same autograd step replayed from a CUDA graph")
    fused = entry(ms_vg, "rmsd_value_and_grad into preallocated outputs, one kernel, replayed from a CUDA graph")
    fused_call = entry(ms_vg_call, "rmsd_value_and_grad called eagerly from Python (allocates its outputs)")
    return {"metric": "RMSD forward+backward atom-frames/s", "unit": "atom-frames/s", "n_frames": F, "n_atoms": n,
            "value": fused["value"], "ms": ms_vg, "l2": "flushed before each step (256 MB write)",
            "roofline": fused["roofline"], "autograd_eager": eager, "autograd_graph": graphed,
            "value_and_grad": fused, "value_and_grad_eager_call": fused_call,
            "max_abs_diff_grad_graph_vs_eager": graph_diff, "max_abs_diff_grad_fused_vs_autograd": vg_diff,
            "oracle_16_frames": {"max_abs_err_rmsd_A": rerr, "max_rel_err_grad": gerr}, "finite": ok}


def run_batched(args, ctx, stream, rank):
    """Batched uneven workload: 512 trajectories, atoms log-uniform in
    50-20,000, frames uniform in 100-5,000, sigma U(0.1, 1.0) A each; forward
    + gradients.  The batched launch (tile shape picked by timing, replayed
    from a CUDA graph) against one forward + one backward call per trajectory
    through the same library (wmd_rmsd_forward / wmd_rmsd_backward)."""
    import numpy as np
    import torch

    from warp_md import _native as N
    from warp_md import synth
    from warp_md.batched import BatchedRmsd

    rng = np.random.default_rng(2024 + rank)
    T = args.batch_traj
    atoms = np.exp(rng.uniform(np.log(50), np.log(20000), T)).astype(np.int64)
    frames = rng.integers(100, 5001, T).astype(np.int64)
    if args.batch_frame_scale != 1.0:
        frames = np.maximum(1, (frames * args.batch_frame_scale).astype(np.int64))
    sig = rng.uniform(0.1, 1.0, T)
    xs, ys = [], []
    for k in range(T):
        x, y = synth.make_trajectory_torch(int(atoms[k]), int(frames[k]), float(sig[k]), seed=100_000 + 1000 * rank + k,
                                           device="cuda", chunk=max(1, (64 << 20) // (24 * int(atoms[k]))))
        xs.append(x)
        ys.append(y)
    units = float((atoms * frames).sum())
    b = BatchedRmsd(xs, ys, with_grad=True)
    g = b.graph()
    for _ in range(max(3, args.warmup)):
        g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.batch_steps):
        g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1) / args.batch_steps
    got = [r.clone() for r in b.rmsd]
    gsample = [gr[: min(4, gr.shape[0])].clone() for gr in b.grads]

    # one forward + one backward launch sequence per trajectory
    refs = [N.Reference(ctx, y.data_ptr(), y.shape[0], 3, keepalive=y) for y in ys]
    outs = [torch.empty(x.shape[0], dtype=torch.float64, device="cuda") for x in xs]
    stats = [torch.empty(x.shape[0], N.FRAME_STATS, dtype=torch.float64, device="cuda") for x in xs]
    ones = [torch.ones(x.shape[0], dtype=torch.float32, device="cuda") for x in xs]
    grads = b.grads

    def loop():
        for k in range(T):
            x = xs[k]
            ctx.check(ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), x.shape[0], x.shape[1], 3, None, x.shape[1],
                                               refs[k].handle, outs[k].data_ptr(), stats[k].data_ptr(),
                                               stream.cuda_stream))
            ctx.check(ctx.lib.wmd_rmsd_backward(ctx.handle, x.data_ptr(), x.shape[0], x.shape[1], 3, None,
                                                x.shape[1], refs[k].handle, stats[k].data_ptr(), ones[k].data_ptr(),
                                                grads[k].data_ptr(), stream.cuda_stream))

    for _ in range(2):
        loop()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.batch_steps):
        loop()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_l = e0.elapsed_time(e1) / args.batch_steps
    d_rmsd = max(float((a - o).abs().max().item()) for a, o in zip(got, outs))
    d_grad = max(float((a - gr[: a.shape[0]]).abs().max().item() / max(1e-30, gr[: a.shape[0]].abs().max().item()))
                 for a, gr in zip(gsample, grads))
    # oracle on the first frames of the two smallest trajectories
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    o_err = 0.0
    for k in np.argsort(atoms)[:2]:
        m = min(50, int(frames[k]))
        _, r64 = oracle.rmsd_frames(xs[k][:m].cpu().numpy(), ys[k].cpu().numpy())
        o_err = max(o_err, float(np.abs(got[k][:m].cpu().numpy() - r64).max()))
    peak, _ = _measured_peaks()
    alg = 36.0 * units + 8.0 * float(frames.sum())
    res = {"metric": "RMSD forward+backward atom-frames/s", "unit": "atom-frames/s", "n_traj": T,
           "atom_frames": units, "frames": int(frames.sum()),
           "batched": {"ms": ms_b, "value": units / (ms_b / 1e3), "layout": b.layout(),
                       "launch": "CUDA graph replay of wmd_batched_rmsd"},
           "per_trajectory": {"ms": ms_l, "value": units / (ms_l / 1e3),
                              "launch": f"{T} x (wmd_rmsd_forward + wmd_rmsd_backward), eager"},
           "speedup_batched_vs_per_trajectory": ms_l / ms_b,
           "roofline": {"bound": "hbm", "achieved": alg / (ms_b / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (ms_b / 1e3) / 1e9 / peak,
                        "note": "36 B/atom-frame: coordinates read by forward and backward, gradient written"},
           "max_abs_diff_rmsd_batched_vs_per_trajectory_A": d_rmsd,
           "max_rel_diff_grad_batched_vs_per_trajectory": d_grad,
           "max_abs_err_vs_oracle_A": o_err, "l2": "inputs larger than L2 (%.0f GB)" % (units * 12 / 1e9)}
    for r in refs:
        r.close()
    del g
    b.close()
    del xs, ys, outs, stats, ones, grads, b, got, gsample
    torch.cuda.empty_cache()
    return res


def run_superpose(args, ctx, stream, rank):
    """SuperposePlan workload: 100,000-atom frames x 2,000 frames (2.4 GB in,
    2.4 GB out), a mass-weighted 10,000-atom selection (every 10th atom) fitted
    to the topology reference, then every atom moved.  Device-resident timing
    of wmd_superpose (statistics, transforms, apply) plus an end-to-end run
    through pinned host buffers; checked against the oracle on sampled frames."""
    import numpy as np
    import torch

    from warp_md import _native as N
    from warp_md import synth

    n_atoms, F = 100_000, args.sp_frames
    x, ref = synth.make_trajectory_torch(n_atoms, F, (0.05, 3.0), seed=40 + rank, device="cuda")
    sel = np.arange(0, n_atoms, 10, dtype=np.uint32)
    rng = np.random.default_rng(5)
    masses = rng.choice(np.array([1.008, 12.011, 14.007, 15.999, 32.06], np.float32), n_atoms)
    ref_h = ref.cpu().numpy()
    r = N.Reference.from_numpy(ctx, ref_h[sel], weights=masses[sel])
    dsel = torch.from_numpy(sel.astype(np.int32)).cuda()
    out = torch.empty(F, n_atoms, 3, device="cuda")
    xf = torch.empty(F, 12, device="cuda")

    def step():
        ctx.check(ctx.lib.wmd_superpose(ctx.handle, x.data_ptr(), F, n_atoms, 3, dsel.data_ptr(), sel.size, r.handle,
                                        0, out.data_ptr(), xf.data_ptr(), stream.cuda_stream))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.sp_steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.sp_steps
    # check sampled frames against the oracle
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    sample = np.arange(0, F, max(1, F // 8))
    host_x = x[sample].cpu().numpy()
    oxf, oout = oracle.superpose(host_x, ref_h[sel], selection=sel, weights=masses[sel])
    got = out[sample].cpu().numpy()
    err_xyz = float(np.abs(got - oout).max())
    err_rot = float(np.abs(xf[sample].cpu().numpy()[:, :9] - oxf[:, :9]).max())
    # end to end: pinned host input and output, copies inside the call
    e2e = None
    try:
        ef = min(F, args.sp_e2e_frames)
        hin = torch.empty(ef, n_atoms, 3, pin_memory=True)
        hin.copy_(x[:ef])
        hout = torch.empty(ef, n_atoms, 3, pin_memory=True)
        hxf = torch.empty(ef, 12, pin_memory=True)

        def e2e_step():
            ctx.check(ctx.lib.wmd_superpose(ctx.handle, hin.data_ptr(), ef, n_atoms, 3, N.ptr(sel), sel.size,
                                            r.handle, 0, hout.data_ptr(), hxf.data_ptr(), stream.cuda_stream))

        e2e_step()
        t0 = time.perf_counter()
        e2e_step()
        dt = time.perf_counter() - t0
        e2e = {"value": float(n_atoms) * ef / dt, "unit": "atom-frames/s", "frames": ef,
               "h2d_bytes_per_step": int(ef * n_atoms * 12), "d2h_bytes_per_step": int(ef * n_atoms * 12 + ef * 48),
               "host_buffer": "pinned", "timing": "host wall clock around the synchronous call"}
        del hin, hout, hxf
    except RuntimeError as exc:
        e2e = {"value": None, "error": str(exc)[:200]}
    peak, _ = _measured_peaks()
    alg = F * (sel.size * 12.0 + n_atoms * 24.0)
    res = {"metric": "superposed atom-frames/s", "unit": "atom-frames/s", "n_atoms": n_atoms, "n_frames": F,
           "n_sel": int(sel.size), "weights": "masses", "ms": ms, "value": n_atoms * F / (ms / 1e3),
           "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (ms / 1e3) / 1e9 / peak,
                        "note": "12 B per selected atom-frame (statistics) + 24 B per atom-frame (read + write)"},
           "max_abs_err_xyz_vs_oracle_A": err_xyz, "max_abs_err_rotation_vs_oracle": err_rot, "e2e": e2e}
    r.close()
    del x, out, xf, dsel
    torch.cuda.empty_cache()
    return res


def run_fluct(args, ctx, stream, rank):
    """RmsfPlan and RmsdPerResPlan workloads on 100,000-atom frames x 2,000
    frames (2.4 GB, device-resident): per-atom RMSF + ADP moments over all
    atoms; per-residue RMSD of 10,000 ten-atom residues after superposing a
    10,000-atom selection.  Checked against the oracle on a sample."""
    import numpy as np
    import torch

    from warp_md import _native as N
    from warp_md import synth

    n_atoms, F = 100_000, args.fl_frames
    x, ref = synth.make_trajectory_torch(n_atoms, F, (0.05, 3.0), seed=60 + rank, device="cuda")
    r = torch.empty(n_atoms, device="cuda")
    a = torch.empty(n_atoms, 6, device="cuda")
    peak, _ = _measured_peaks()

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def rmsf_step():
        ctx.check(ctx.lib.wmd_rmsf(ctx.handle, x.data_ptr(), F, n_atoms, 3, None, n_atoms, r.data_ptr(), a.data_ptr(),
                                   stream.cuda_stream))

    ms_f = timed(rmsf_step, args.fl_steps)
    # per-residue RMSD: residues of 10 consecutive atoms, every 10th atom selected
    sel = np.arange(0, n_atoms, 10, dtype=np.uint32)
    goff = np.arange(0, n_atoms + 1, 10, dtype=np.uint32)
    gat = np.arange(n_atoms, dtype=np.uint32)
    n_groups = goff.size - 1
    ref_h = ref.cpu().numpy()
    rr = N.Reference.from_numpy(ctx, ref_h[sel])
    dsel = torch.from_numpy(sel.astype(np.int32)).cuda()
    groups_ref = N.GroupRef(ctx, ref_h, goff, gat)
    out = torch.empty(F, n_groups, device="cuda")

    def perres_step():
        ctx.check(ctx.lib.wmd_rmsd_per_group(ctx.handle, x.data_ptr(), F, n_atoms, 3, dsel.data_ptr(), sel.size,
                                             rr.handle, groups_ref.handle, 1, out.data_ptr(), stream.cuda_stream))

    ms_p = timed(perres_step, args.fl_steps)
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    sample = slice(0, min(F, 64))
    hx = x[sample].cpu().numpy()
    keep = np.arange(0, n_atoms, 101)
    orr, _ = oracle.rmsf(x.cpu().numpy()[:, keep])
    err_rmsf = float(np.abs(r.cpu().numpy()[keep] - orr).max())
    groups = [np.arange(g * 10, g * 10 + 10) for g in range(0, n_groups, 97)]
    want = oracle.rmsd_perres(hx, ref_h, groups, selection=sel, align=True)
    got = out[sample].cpu().numpy()[:, ::97]
    err_pr = float(np.abs(got - want).max())
    alg_f = 12.0 * n_atoms * F
    alg_p = F * (12.0 * sel.size + 12.0 * n_atoms + 4.0 * n_groups)
    res = {"rmsf": {"metric": "RMSF atom-frames/s", "unit": "atom-frames/s", "n_atoms": n_atoms, "n_frames": F,
                    "ms": ms_f, "value": n_atoms * F / (ms_f / 1e3),
                    "roofline": {"bound": "hbm", "achieved": alg_f / (ms_f / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                                 "frac": alg_f / (ms_f / 1e3) / 1e9 / peak, "note": "12 B per atom-frame"},
                    "max_abs_err_vs_oracle_A": err_rmsf, "outputs": "RMSF + 6 ADP moments per atom"},
           "rmsd_perres": {"metric": "per-residue RMSD atom-frames/s", "unit": "atom-frames/s", "n_atoms": n_atoms,
                           "n_frames": F, "n_residues": n_groups, "n_sel": int(sel.size), "ms": ms_p,
                           "value": n_atoms * F / (ms_p / 1e3),
                           "roofline": {"bound": "hbm", "achieved": alg_p / (ms_p / 1e3) / 1e9, "peak": peak,
                                        "unit": "GB/s", "frac": alg_p / (ms_p / 1e3) / 1e9 / peak,
                                        "note": "12 B per selected atom-frame + 12 B per atom-frame + 4 B per "
                                                "residue-frame"},
                           "max_abs_err_vs_oracle_A": err_pr}}
    rr.close()
    groups_ref.close()
    del x, r, a, out, dsel
    torch.cuda.empty_cache()
    return res


def run_cluster(args, ctx, stream, rank):
    """TrajectoryClusterPlan workloads on the all-pairs trajectory (20,000
    frames x 1,000 atoms): DBSCAN over the tensor-core (i8x3) matrix and over
    the FP64 matrix, and k-means (8 clusters, 20 iterations) on the frames
    superposed onto frame 0.  Device-resident inputs; checked against the
    oracle on a 1,000-frame prefix."""
    import ctypes

    import numpy as np
    import torch

    from warp_md import _native as N
    from warp_md import synth
    from warp_md.plans import _PAIR_MODES

    F, n = args.cl_frames, PAIR_ATOMS
    coords = synth.make_drift_trajectory_torch(n, F, 0.1, seed=3 + rank, device="cuda")
    labels = torch.empty(F, dtype=torch.int32, device="cuda")
    cent = torch.empty(F, dtype=torch.int32, device="cuda")
    sizes = torch.empty(F, dtype=torch.int32, device="cuda")
    k = ctypes.c_int64(0)
    eps = 1.0

    def dbscan(mode):
        ctx.check(ctx.lib.wmd_cluster_dbscan(ctx.handle, coords.data_ptr(), F, n, 3, None, n, _PAIR_MODES[mode], eps,
                                             5, labels.data_ptr(), cent.data_ptr(), sizes.data_ptr(),
                                             ctypes.byref(k), stream.cuda_stream))

    def kmeans():
        ctx.check(ctx.lib.wmd_cluster_kmeans(ctx.handle, coords.data_ptr(), F, n, 3, None, n, 8, 20, 0.0, 7,
                                             labels.data_ptr(), cent.data_ptr(), sizes.data_ptr(), ctypes.byref(k),
                                             stream.cuda_stream))

    res = {"n_frames": F, "n_atoms": n, "workload": PAIR_WORKLOAD}

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps * 1e3

    for mode in ("i8x3", "fp64"):
        ms = timed(lambda: dbscan(mode), 1 if mode == "fp64" else 3)
        res[f"dbscan_{mode}"] = {"ms": ms, "n_clusters": int(k.value), "eps": eps, "min_samples": 5,
                                 "noise": int((labels == -1).sum().item()),
                                 "timing": "host wall clock around the synchronous call (matrix + DBSCAN)"}
    ms = timed(kmeans, 1)
    res["kmeans"] = {"ms": ms, "n_clusters": 8, "iterations": 20, "sizes": sizes[: int(k.value)].cpu().tolist()}
    # parity on a prefix
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle

    m = min(F, 1000)
    host = coords[:m].cpu().numpy()
    d32, _ = oracle.pairwise(host)
    ol, oc, osz = oracle.dbscan(d32, eps, 5)
    sub = coords[:m].contiguous()
    ctx.check(ctx.lib.wmd_cluster_dbscan(ctx.handle, sub.data_ptr(), m, n, 3, None, n, _PAIR_MODES["fp64"], eps, 5,
                                         labels.data_ptr(), cent.data_ptr(), sizes.data_ptr(), ctypes.byref(k),
                                         stream.cuda_stream))
    res["dbscan_parity_1000"] = bool(np.array_equal(labels[:m].cpu().numpy(), ol) and
                                     np.array_equal(cent[: int(k.value)].cpu().numpy().astype(np.uint32), oc))
    del coords, labels, cent, sizes
    torch.cuda.empty_cache()
    return res


def _write_dcd(path, coords, cell=100.0, chunk=100):
    """A little-endian DCD (4-byte markers, CHARMM header) with an
    orthorhombic unit-cell record per frame, written chunk by chunk from a CUDA
    tensor [F][N][3]: the record layout warp-md's DcdWriter produces
    (crates/traj-io/src/dcd.rs:573-708)."""
    import struct

    import numpy as np

    F, n = coords.shape[0], coords.shape[1]
    icntrl = [0] * 20
    icntrl[0], icntrl[10], icntrl[19] = F, 1, 24

    def rec(payload):
        return struct.pack("<I", len(payload)) + payload + struct.pack("<I", len(payload))

    head = (rec(b"CORD" + struct.pack("<20i", *icntrl)) + rec(struct.pack("<i", 1) + b"WARP_MD_B200_BENCH".ljust(80))
            + rec(struct.pack("<i", n)))
    cellrec = rec(np.array([cell, 0.0, cell, 0.0, 0.0, cell], "<f8").tobytes())
    with open(path, "wb") as fh:
        fh.write(head)
        for f0 in range(0, F, chunk):
            xyz = coords[f0:f0 + chunk].transpose(1, 2).contiguous().cpu().numpy()  # [f][3][n]
            body = np.empty((xyz.shape[0], 3, n + 2), np.uint32)
            body[:, :, 0] = body[:, :, -1] = 4 * n
            body[:, :, 1:-1] = xyz.view(np.uint32)
            cells = np.frombuffer(cellrec, np.uint8)
            out = np.empty((xyz.shape[0], cells.size + body[0].nbytes), np.uint8)
            out[:, :cells.size] = cells
            out[:, cells.size:] = body.reshape(xyz.shape[0], -1).view(np.uint8)
            out.tofile(fh)


def _scratch_dir(need_bytes):
    import shutil
    import tempfile

    for cand in ("/dev/shm", tempfile.gettempdir(), HERE):
        try:
            if shutil.disk_usage(cand).free > 2 * need_bytes:
                return tempfile.mkdtemp(prefix="wmd_dcd_", dir=cand)
        except OSError:
            continue
    return None


def run_dcd(args, ctx, stream, rank):
    """RmsdPlan over a DCD file (100,000 atoms x --dcd-frames frames, unit
    cells, written here and read back from the page cache): the file read
    (threaded pread into pinned buffers), the copy, the GPU decode and the RMSD
    kernels overlapped by wmd_dcd_rmsd; host wall clock around the synchronous
    call.  Also: the file decoded into device memory (wmd_dcd_read), a pinned
    host->device copy for scale, and the oracle reader + RMSD on a bounded
    sample of the same file format."""
    import shutil

    import numpy as np
    import torch

    import warp_md
    from warp_md import synth

    F, n = args.dcd_frames, N_ATOMS
    frame_bytes = 3 * (4 * n + 8) + 56
    d = _scratch_dir(F * frame_bytes)
    if d is None:
        return {"error": "no scratch space for the trajectory file"}
    try:
        coords, ref = synth.make_trajectory_torch(n, F, SIGMA, seed=31 + rank, device="cuda")
        path = os.path.join(d, "bench.dcd")
        _write_dcd(path, coords)
        ref_np = ref.cpu().numpy()
        system = warp_md.System.from_arrays({"name": ["CA"] * n, "resid": list(range(1, n + 1))}, positions0=ref_np)
        traj = warp_md.Trajectory.open_dcd(path, system)
        size = os.path.getsize(path)

        def timed(fn, reps):
            # median of individually timed calls: the host side (page cache,
            # pread threads) shares the machine's cores and memory with other jobs
            for _ in range(max(1, args.warmup)):
                fn()
            torch.cuda.synchronize()
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                fn()
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t0)
            return statistics.median(ts)

        out = {}

        def rmsd_step():
            out["v"] = traj.rmsd(ref_np)

        sec = timed(rmsd_step, args.dcd_steps)
        dev = torch.empty((F, n, 3), dtype=torch.float32, device="cuda")

        def read_step():
            traj.read_device(0, F, out=dev)

        sec_read = timed(read_step, args.dcd_steps)
        ok_read = bool(torch.equal(dev, coords))
        del dev
        torch.cuda.empty_cache()
        # pinned host -> device copy of 1 GiB, the link's rate
        pin = torch.empty(1 << 28, dtype=torch.float32, pin_memory=True)
        dst = torch.empty_like(pin, device="cuda")
        sec_h2d = timed(lambda: dst.copy_(pin, non_blocking=True), 5)
        del pin, dst
        # parity of the first frames against the oracle's reader and RMSD
        sys.path.insert(0, os.path.join(HERE, "oracle"))
        import dcd_oracle
        import oracle

        m = min(F, args.dcd_cpu_frames)
        sub = os.path.join(d, "sample.dcd")
        _write_dcd(sub, coords[:m])
        t0 = time.perf_counter()
        cframes = dcd_oracle.read_all(sub, needs_box=False)[0]
        cvals = oracle.rmsd_frames(cframes, ref_np, threads=1)[1]
        cpu_sec = time.perf_counter() - t0
        err = float(np.abs(out["v"][:m] - cvals).max())
        res = {
            "workload": f"DCD file of {F} frames x {n} atoms with unit cells ({size / 1e9:.2f} GB, page cache)",
            "rmsd_from_file": {"seconds": sec, "value": n * F / sec, "unit": UNIT, "file_gbs": size / sec / 1e9,
                               "timing": "median host wall clock around wmd_dcd_rmsd (pread + H2D + decode + RMSD)",
                               "pread_threads": int(os.environ.get("WMD_DCD_THREADS", "0")) or min(16, os.cpu_count() or 1)},
            "read_to_device": {"seconds": sec_read, "file_gbs": size / sec_read / 1e9, "bit_exact": ok_read},
            "h2d_pinned_gbs": (1 << 30) / sec_h2d / 1e9,
            "cpu_reader_rmsd": {"value": n * m / cpu_sec, "unit": UNIT, "frames": m, "seconds": cpu_sec,
                                "kind": "port", "cores": 1,
                                "sample": f"first {m} frames: oracle sequential reader + FP64 RMSD, 1 thread"},
            "max_abs_err_vs_oracle_A": err,
        }
        traj.close()
        del coords
        torch.cuda.empty_cache()
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_reference(args):
    """The reference's CPU path for the headline workload: the oracle port of
    rmsd_aligned_selected (no build of the Rust reference is possible here) on
    all host threads, statically scheduled so every thread gets an equal run of
    frames.  One sample of frames is generated once; every step times one pass
    over it.  The reference path itself is single-threaded, so a 1-thread pass
    over a smaller sample is reported beside it."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle
    from warp_md import synth

    threads = os.cpu_count() or 1
    frames = args.ref_frames
    fr, ref = synth.make_trajectory(N_ATOMS, frames, SIGMA, seed=100)
    vals = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.rmsd_frames(fr, ref, threads=threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            vals.append(N_ATOMS * frames / dt)
    value = statistics.median(vals)
    one = max(2, min(args.ref_frames_single, frames))
    t0 = time.perf_counter()
    oracle.rmsd_frames(fr[:one], ref, threads=1)
    dt_one = time.perf_counter() - t0
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": N_ATOMS * frames / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": N_ATOMS, "n_frames": N_FRAMES, "sample_frames": frames},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"the same {frames} frames x {N_ATOMS} atoms of the workload every step, "
                                    f"OpenMP static schedule over {threads} threads"),
                         "single_thread": {"value": N_ATOMS * one / dt_one, "frames": one, "seconds": dt_one,
                                           "note": "the reference's RmsdPlan CPU path runs on one thread"}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _r(v, digits=4):
    """Rounds to `digits` significant digits (compact JSON)."""
    if v is None:
        return None
    return float(f"{v:.{digits}g}")


def _summary(pairwise, differentiable, batched, odd=None):
    """The pairwise (plain vs mixed), differentiable and batched figures in a
    few hundred characters."""
    out = {}
    if odd:
        out["frames_99999_atoms"] = {"ms": _r(odd["ms"]), "hbm_frac": _r(odd["roofline"]["frac"], 3)}
    if pairwise:
        p = {"metric": "2D-RMSD pairs/s at <=1e-4 A, plain FP32 vs tensor int8 limbs",
             "frames": pairwise["n_frames"], "atoms": pairwise["n_atoms"], "err_block": "512x512 vs FP64 oracle"}
        for m in ("fp32", "i8x3", "i8x2"):
            e = pairwise.get(m)
            if e:
                p[m] = {"ms": _r(e["ms"]), "pairs_s": _r(e["value"]), "max_err_A": _r(e["max_err_A"], 2),
                        "rms_err_A": _r(e["rms_err_A"], 2)}
                if "roofline" in e:
                    p[m]["tensor_frac"] = _r(e["roofline"]["frac"], 3)
        for k in ("speedup_i8x3_vs_fp32", "speedup_i8x2_vs_fp32"):
            if k in pairwise:
                p[k] = _r(pairwise[k], 3)
        out["pairwise"] = p
    if differentiable:
        d = differentiable
        out["differentiable"] = {
            "bytes_per_af": 24,
            "value_and_grad": {"ms": _r(d["value_and_grad"]["ms"]), "hbm_frac": _r(d["value_and_grad"]["roofline"]["frac"], 3)},
            "autograd_graph": {"ms": _r(d["autograd_graph"]["ms"]), "hbm_frac": _r(d["autograd_graph"]["roofline"]["frac"], 3)},
            "autograd_eager": {"ms": _r(d["autograd_eager"]["ms"]), "hbm_frac": _r(d["autograd_eager"]["roofline"]["frac"], 3)},
            "oracle_err": [_r(d["oracle_16_frames"]["max_abs_err_rmsd_A"], 2), _r(d["oracle_16_frames"]["max_rel_err_grad"], 2)]}
    if batched:
        b = batched
        out["batched_uneven"] = {"ms": _r(b["batched"]["ms"]), "af_s": _r(b["batched"]["value"]),
                                 "hbm_frac": _r(b["roofline"]["frac"], 3),
                                 "per_traj_ms": _r(b["per_trajectory"]["ms"]),
                                 "oracle_err_A": _r(b["max_abs_err_vs_oracle_A"], 2)}
    return out


def run_ours(args):
    import numpy as np
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    from warp_md import _native as N
    from warp_md import synth

    ctx = N.context(local)
    stream = torch.cuda.current_stream()
    n_frames = args.n_frames
    coords, ref = synth.make_trajectory_torch(N_ATOMS, n_frames, SIGMA, seed=1 + rank, device="cuda")
    r = N.Reference(ctx, ref.data_ptr(), N_ATOMS, 3, keepalive=ref)
    out = torch.empty(n_frames, dtype=torch.float64, device="cuda")

    def step():
        ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, coords.data_ptr(), n_frames, N_ATOMS, 3, None, N_ATOMS,
                                          r.handle, 1, out.data_ptr(), stream.cuda_stream))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        step()
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    per_launch_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if pg:
        t = torch.tensor([total_ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
        pg.barrier()
    units = float(N_ATOMS) * n_frames * ws * args.steps
    value = units / (total_ms / 1e3)
    kern_ms = statistics.median(per_launch_ms)
    alg_bytes = N_ATOMS * n_frames * BYTES_PER_UNIT + n_frames * BYTES_PER_FRAME_OUT
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    peak, peak_kind = _measured_peaks()
    traffic = None
    tfile = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as fh:
            tj = json.load(fh)
        if "rmsd_frames_bytes_per_atom_frame" in tj:
            traffic = tj["rmsd_frames_bytes_per_atom_frame"] * N_ATOMS * n_frames

    # sanity: results finite, a sample against nothing but physics (rmsd within noise range)
    vals = out.cpu().numpy()
    assert np.all(np.isfinite(vals)), "non-finite RMSD"

    # the same buffer as 99,999-atom frames: a frame stride that is not a
    # multiple of 16 bytes (the frames-across-lanes kernel on quad rows)
    odd = None
    if rank == 0:
        n_odd = N_ATOMS - 1
        xo = coords.view(-1)[: n_frames * n_odd * 3].view(n_frames, n_odd, 3)
        ro_t = ref[:n_odd].contiguous()
        ro = N.Reference(ctx, ro_t.data_ptr(), n_odd, 3, keepalive=ro_t)
        oo = torch.empty(n_frames, dtype=torch.float64, device="cuda")

        def odd_step():
            ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, xo.data_ptr(), n_frames, n_odd, 3, None, n_odd, ro.handle,
                                              1, oo.data_ptr(), stream.cuda_stream))

        for _ in range(3):
            odd_step()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            odd_step()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms_odd = statistics.median(ts)
        ach = (n_odd * n_frames * BYTES_PER_UNIT + n_frames * BYTES_PER_FRAME_OUT) / (ms_odd / 1e3) / 1e9
        odd = {"n_atoms": n_odd, "n_frames": n_frames, "ms": ms_odd, "value": n_odd * n_frames / (ms_odd / 1e3),
               "roofline": {"bound": "hbm", "achieved": ach, "peak": _measured_peaks()[0], "unit": "GB/s",
                            "frac": ach / _measured_peaks()[0]},
               "note": "the headline buffer read as 99,999-atom frames (frame stride not a multiple of 16 bytes)"}
        assert bool(torch.isfinite(oo).all().item())
        ro.close()
        del xo, oo, ro_t

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    host = None
    if not args.skip_e2e:
        e2e_frames = n_frames
        try:
            host = torch.empty((e2e_frames, N_ATOMS, 3), dtype=torch.float32, pin_memory=True)
            host.copy_(coords[:e2e_frames])
            hout = np.empty(e2e_frames, np.float64)

            def e2e_step():
                ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, host.data_ptr(), e2e_frames, N_ATOMS, 3, None,
                                                  N_ATOMS, r.handle, 1, hout.ctypes.data, stream.cuda_stream))

            e2e_step()
            torch.cuda.synchronize()
            if pg:
                pg.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(max(1, args.e2e_steps)):
                e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            ems = e0.elapsed_time(e1)
            if pg:
                t = torch.tensor([ems], device="cuda")
                pg.all_reduce(t, op=pg.ReduceOp.MAX)
                ems = float(t.item())
            e2e = {"value": float(N_ATOMS) * e2e_frames * ws * max(1, args.e2e_steps) / (ems / 1e3), "unit": UNIT,
                   "h2d_bytes_per_step": int(e2e_frames * N_ATOMS * 12), "d2h_bytes_per_step": int(e2e_frames * 8),
                   "frames": e2e_frames, "host_buffer": "pinned"}
            # host input runs in chunks whose launches may tile the atoms
            # differently; the FP64 sums then round differently (~1e-8 A here)
            e2e_diff = float(np.abs(hout - vals[:e2e_frames]).max())
            assert e2e_diff <= 1e-6, e2e_diff
            e2e["max_abs_diff_vs_device_resident_A"] = e2e_diff
        except RuntimeError as exc:  # e.g. pinned allocation refused on the host
            e2e = {"value": None, "unit": UNIT, "error": str(exc)[:200]}

    cpu = None
    if rank == 0 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        if host is not None:
            hframes, href = host.numpy(), ref.cpu().numpy()
        else:
            hframes, href = None, None
        all_frames = min(args.cpu_frames, n_frames) if hframes is not None else args.cpu_frames
        v_all, dt_all, cvals = cpu_baseline(threads, all_frames, frames=hframes, ref=href)
        one_frames = max(2, min(args.cpu_frames_single, all_frames))
        v_one, dt_one, _ = cpu_baseline(1, one_frames, frames=hframes, ref=href)
        err = None
        if hframes is not None:
            err = float(np.abs(cvals - vals[:all_frames]).max())
        cpu = {"value": v_all, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"first {all_frames} frames x {N_ATOMS} atoms of the workload "
                          f"({dt_all:.1f} s with {threads} threads)"),
               "single_thread": {"value": v_one, "frames": one_frames, "seconds": dt_one},
               "max_abs_err_gpu_vs_cpu_A": err}
    del host, coords, out
    torch.cuda.empty_cache()

    pairwise = None
    if not args.skip_pairwise:
        pairwise = run_pairwise(args, ctx, stream, rank)
    differentiable = None
    if not args.skip_diff:
        differentiable = run_differentiable(args, stream, rank)
    batched = None
    if not args.skip_batched:
        batched = run_batched(args, ctx, stream, rank)
    superpose = None
    if not args.skip_superpose:
        superpose = run_superpose(args, ctx, stream, rank)
    fluct = None
    if not args.skip_fluct:
        fluct = run_fluct(args, ctx, stream, rank)
    cluster = None
    if not args.skip_cluster:
        cluster = run_cluster(args, ctx, stream, rank)
    dcd = None
    if not args.skip_dcd:
        dcd = run_dcd(args, ctx, stream, rank)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_atoms": N_ATOMS, "n_frames_per_gpu": n_frames,
                       "input_layout": "float32 xyz, frame-major", "l2": "inputs larger than L2 (12 GB per GPU)",
                       "parallelism": f"frames sharded, {ws} independent ranks"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "kernel": "wmd::rmsd_lanes_kernel (frames across lanes) + rmsd_finalize_kernel (QCP)",
                         "kernel_ms": kern_ms,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
            "frames_odd_atoms": odd,
            "superpose": superpose,
            "fluct": fluct,
            "cluster": cluster,
            "dcd": dcd,
            "pairwise": pairwise,
            "differentiable": differentiable,
            "batched_uneven": batched,
            # last, so that a reader that keeps only the end of the line still
            # has the second half of the metric
            "summary": _summary(pairwise, differentiable, batched, odd),
        }
        print(json.dumps(line), flush=True)
    r.close()
    if pg:
        pg.destroy_process_group()
    return 0


def run_profile_case(name):
    """Small cases of single kernels for ncu captures (``--profile-case``); they
    print no bench line.

    vg:   4,096 frames x 2,000 atoms through wmd_rmsd_forward,
          wmd_rmsd_backward_f64 and wmd_rmsd_value_and_grad, twice, with a
          256 MB write (larger than L2) before the forward and the fused call.
    quad: 99,999-atom frames (a 12-byte frame stride that is not a multiple of
          16 bytes: quad rows) x 400 frames through wmd_rmsd_frames, 3 calls.
    perres: per-residue RMSD of 100,000 atoms x 2,000 frames (2.4 GB), residues
          of 10 consecutive atoms, every 10th atom superposed: 3 calls of
          wmd_rmsd_per_group.
    batched: 24 trajectories drawn like the batched workload's (atoms
          log-uniform 50-20,000, frames uniform 50-2,500), lanes layout with
          1,024-atom tiles, forward + gradients, 3 runs.
    """
    import numpy as np
    import torch
    from warp_md import _native as N
    from warp_md import synth

    ctx = N.context(0)
    if name == "vg":
        F, n = 4096, 2000
        fr, rf = synth.make_trajectory(n, F, 0.3, seed=17)
        x = torch.from_numpy(fr).cuda()
        ref = torch.from_numpy(rf).cuda()
        r = N.Reference(ctx, ref.data_ptr(), n, 3, keepalive=ref)
        out = torch.empty(F, dtype=torch.float64, device="cuda")
        stats = torch.empty(F, N.FRAME_STATS, dtype=torch.float64, device="cuda")
        g = torch.empty_like(x)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        for _ in range(2):
            flush.fill_(1)
            ctx.check(ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle,
                                               out.data_ptr(), stats.data_ptr(), None))
            ctx.check(ctx.lib.wmd_rmsd_backward_f64(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle,
                                                    stats.data_ptr(), None, 0, g.data_ptr(), None))
            flush.fill_(1)
            ctx.check(ctx.lib.wmd_rmsd_value_and_grad(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle,
                                                      None, 0, out.data_ptr(), g.data_ptr(), None))
    elif name == "quad":
        n, F = 99_999, 400
        x, ref = synth.make_trajectory_torch(n, F, SIGMA, seed=1, device="cuda")
        r = N.Reference(ctx, ref.data_ptr(), n, 3, keepalive=ref)
        out = torch.empty(F, dtype=torch.float64, device="cuda")
        for _ in range(3):
            ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, 1,
                                              out.data_ptr(), None))
    elif name == "perres":
        n, F = 100_000, 2000
        x, ref = synth.make_trajectory_torch(n, F, SIGMA, seed=3, device="cuda")
        ref_h = ref.cpu().numpy()
        sel = np.arange(0, n, 10, dtype=np.uint32)
        goff = np.arange(0, n + 1, 10, dtype=np.uint32)
        gref = N.GroupRef(ctx, ref_h, goff, np.arange(n, dtype=np.uint32))
        r = N.Reference.from_numpy(ctx, ref_h[sel])
        dsel = torch.from_numpy(sel.astype(np.int32)).cuda()
        out = torch.empty(F, goff.size - 1, device="cuda")
        for _ in range(3):
            ctx.check(ctx.lib.wmd_rmsd_per_group(ctx.handle, x.data_ptr(), F, n, 3, dsel.data_ptr(), sel.size,
                                                 r.handle, gref.handle, 1, out.data_ptr(), None))
        torch.cuda.synchronize()
        gref.close()
    elif name == "batched":
        from warp_md.batched import BatchedRmsd

        os.environ["WARPMD_BATCHED_LAYOUT"] = "lanes"
        os.environ["WARPMD_BATCHED_TILE_ATOMS"] = "1024"
        rng = np.random.default_rng(2024)
        T = 24
        atoms = np.exp(rng.uniform(np.log(50), np.log(20000), T)).astype(np.int64)
        frames = np.maximum(1, rng.integers(100, 5001, T) // 2).astype(np.int64)
        xs, ys = [], []
        for k in range(T):
            x, y = synth.make_trajectory_torch(int(atoms[k]), int(frames[k]), 0.5, seed=100_000 + k, device="cuda",
                                               chunk=max(1, (64 << 20) // (24 * int(atoms[k]))))
            xs.append(x)
            ys.append(y)
        b = BatchedRmsd(xs, ys, with_grad=True)
        for _ in range(3):
            b.run()
        torch.cuda.synchronize()
        b.close()
        r = None
    else:
        raise SystemExit(f"unknown profile case {name!r}")
    torch.cuda.synchronize()
    if r is not None:
        r.close()
    print(f"profile case {name}: ok", flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-frames", type=int, default=10_000)
    ap.add_argument("--cpu-frames-single", type=int, default=1_000)
    ap.add_argument("--n-frames", type=int, default=N_FRAMES, help="frames per GPU (profiling runs only)")
    ap.add_argument("--ref-frames", type=int, default=2000, help="reference arm: frames per timed sample")
    ap.add_argument("--ref-frames-single", type=int, default=300, help="reference arm: frames of the 1-thread pass")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-pairwise", action="store_true")
    ap.add_argument("--pair-frames", type=int, default=20_000)
    ap.add_argument("--pair-steps", type=int, default=3)
    ap.add_argument("--pair-modes", default="fp32,i8x3,i8x2")
    ap.add_argument("--skip-diff", action="store_true")
    ap.add_argument("--diff-steps", type=int, default=20)
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--batch-traj", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--batch-frame-scale", type=float, default=1.0, help="scale frame counts (profiling runs only)")
    ap.add_argument("--skip-superpose", action="store_true")
    ap.add_argument("--sp-frames", type=int, default=2000)
    ap.add_argument("--sp-steps", type=int, default=5)
    ap.add_argument("--sp-e2e-frames", type=int, default=500)
    ap.add_argument("--skip-fluct", action="store_true")
    ap.add_argument("--fl-frames", type=int, default=2000)
    ap.add_argument("--fl-steps", type=int, default=5)
    ap.add_argument("--skip-cluster", action="store_true")
    ap.add_argument("--cl-frames", type=int, default=20_000)
    ap.add_argument("--skip-dcd", action="store_true")
    ap.add_argument("--dcd-frames", type=int, default=2000)
    ap.add_argument("--dcd-steps", type=int, default=5)
    ap.add_argument("--dcd-cpu-frames", type=int, default=100)
    ap.add_argument("--profile-case", choices=["vg", "quad", "perres", "batched"], help="run one small kernel case for ncu and exit")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args.profile_case)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
