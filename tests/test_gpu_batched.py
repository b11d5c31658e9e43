"""Batched launch over many trajectories of uneven size (wmd_batched_prepare /
wmd_batched_rmsd) against the oracle per trajectory and against the
single-trajectory entry points.

The reference has no batched form; each trajectory's values must be what its
own RmsdPlan gives (plan.rs:164-418), so the pins are the oracle's FP64 RMSD
(|d| <= 1e-5 A, the per-frame bar) and its analytic gradient
(|g - g64| <= 1e-5 max|g| + 1e-7).  Every layout (tile-major, frame-major,
tile-major with the frames-across-lanes forward) and both tile shapes (512
and 1024 atoms) are forced once each, and the autotuner's own choice is run
too.
"""
import os

import numpy as np
import pytest

import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# atoms, frames: ragged around both tile sizes, a one-atom-short tail, empty
# trajectories of both kinds, a single frame and a single atom
SHAPES = [(50, 10), (511, 3), (512, 4), (1023, 5), (1024, 2), (1025, 7), (3000, 6), (0, 4), (700, 0),
          (1, 3), (2049, 1), (20000, 3), (7, 13)]


def _batch(shapes, seed, near_zero=()):
    xs, ys = [], []
    for k, (n, F) in enumerate(shapes):
        if n == 0 or F == 0:
            xs.append(np.zeros((F, n, 3), np.float32))
            ys.append(np.zeros((n, 3), np.float32))
            continue
        fr, ref = synth.make_trajectory(n, F, 0.4, seed + k)
        # a reference that is none of the frames, except where RMSD ~ 0 is wanted
        if k not in near_zero:
            ref = (ref + np.random.default_rng(seed + 100 + k).normal(0, 0.3, ref.shape)).astype(np.float32)
        xs.append(fr)
        ys.append(ref)
    return xs, ys


def _run(xs, ys, with_grad, tile=None, layout=None):
    from warp_md.batched import BatchedRmsd

    pins = {"WARPMD_BATCHED_TILE_ATOMS": None if tile is None else str(tile), "WARPMD_BATCHED_LAYOUT": layout}
    old = {k: os.environ.get(k) for k in pins}
    for k, v in pins.items():
        if v is not None:
            os.environ[k] = v
    try:
        b = BatchedRmsd([torch.from_numpy(x).cuda() for x in xs], [torch.from_numpy(y).cuda() for y in ys],
                        with_grad=with_grad)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    if tile is not None:
        assert b.layout()["tile_atoms"] == tile
    if layout is not None:
        assert b.layout()["layout"] == layout
        assert b.layout()["frame_major"] == (layout == "frames")
    for r in b.rmsd:
        r.fill_(-1.0)
    b.run()
    torch.cuda.synchronize()
    return b


def _check_rmsd(b, xs, ys):
    for k, (x, y) in enumerate(zip(xs, ys)):
        got = b.rmsd[k].cpu().numpy()
        if x.shape[0] == 0:
            assert got.size == 0
            continue
        if x.shape[1] == 0:
            np.testing.assert_array_equal(got, 0.0)
            continue
        _, r64 = oracle.rmsd_frames(x, y)
        err = np.abs(got - r64).max()
        assert err <= 1e-5, (k, x.shape, err)


def _check_grad(b, xs, ys):
    for k, (x, y) in enumerate(zip(xs, ys)):
        if x.size == 0:
            continue
        _, g = oracle.rmsd_grad(x, y)
        got = b.grads[k].cpu().numpy()
        tol = 1e-5 * np.abs(g).max() + 1e-7
        err = np.abs(got - g).max()
        assert err <= tol, (k, x.shape, err, tol)


LAYOUTS = [(512, "tiles"), (1024, "tiles"), (512, "frames"), (1024, "frames"), (512, "lanes"), (1024, "lanes"),
           (None, None)]


@pytest.mark.parametrize("tile,layout", LAYOUTS)
def test_batched_forward_matches_oracle(tile, layout):
    xs, ys = _batch(SHAPES, 11)
    b = _run(xs, ys, with_grad=False, tile=tile, layout=layout)
    _check_rmsd(b, xs, ys)
    b.close()


@pytest.mark.parametrize("tile,layout", LAYOUTS)
def test_batched_gradients_match_oracle(tile, layout):
    xs, ys = _batch(SHAPES, 23)
    b = _run(xs, ys, with_grad=True, tile=tile, layout=layout)
    _check_rmsd(b, xs, ys)
    _check_grad(b, xs, ys)
    b.close()


def test_batched_equals_single_trajectory_path():
    """Each trajectory's values equal torch_ops.rmsd (wmd_rmsd_forward /
    wmd_rmsd_backward) on it alone: the same FP64 statistics and QCP, so the
    two differ only by summation order (<= 1e-9 A here)."""
    xs, ys = _batch([(300, 8), (4100, 5), (1024, 9), (77, 30)], 31)
    for layout in ("tiles", "frames", "lanes"):
        _compare_single(_run(xs, ys, with_grad=True, layout=layout), xs, ys)


def _compare_single(b, xs, ys):
    from warp_md.torch_ops import rmsd

    for k, (x, y) in enumerate(zip(xs, ys)):
        xt = torch.from_numpy(x).cuda().requires_grad_(True)
        v = rmsd(xt, torch.from_numpy(y).cuda())
        v.sum().backward()
        np.testing.assert_allclose(b.rmsd[k].cpu().numpy(), v.detach().cpu().numpy(), rtol=0, atol=1e-9)
        g1, g2 = b.grads[k].cpu().numpy(), xt.grad.cpu().numpy()
        assert np.abs(g1 - g2).max() <= 1e-6 * np.abs(g2).max() + 1e-8
    b.close()


def test_batched_near_zero_rmsd_takes_residual_pass():
    """Trajectories whose frames are rigid motions of the reference: RMSD is
    the float32 rounding level and must still match the oracle to 1e-5 A."""
    shapes = [(2000, 6), (300, 4), (1500, 3)]
    xs, ys = _batch(shapes, 41, near_zero=(0, 1, 2))
    rng = np.random.default_rng(5)
    for k in range(len(xs)):
        for f in range(xs[k].shape[0]):
            q = rng.normal(size=4)
            q /= np.linalg.norm(q)
            w, x, y, z = q
            R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                          [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                          [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
            xs[k][f] = (ys[k].astype(np.float64) @ R.T + rng.normal(0, 5, 3)).astype(np.float32)
    for layout in ("tiles", "frames", "lanes"):
        b = _run(xs, ys, with_grad=True, layout=layout)
        _check_rmsd(b, xs, ys)
        for r in b.rmsd:
            assert r.max().item() < 1e-3
        for g in b.grads:
            assert torch.isfinite(g).all()
        b.close()


def test_batched_graph_replay_follows_inputs():
    xs, ys = _batch([(900, 5), (60, 12), (2500, 3)], 51)
    from warp_md.batched import BatchedRmsd

    xt = [torch.from_numpy(x).cuda() for x in xs]
    b = BatchedRmsd(xt, [torch.from_numpy(y).cuda() for y in ys], with_grad=True)
    g = b.graph()
    # new coordinates in place, then replay
    xs2, _ = _batch([(900, 5), (60, 12), (2500, 3)], 61)
    for t, x in zip(b.coords, xs2):
        t.copy_(torch.from_numpy(x))
    for r in b.rmsd:
        r.fill_(-1.0)
    g.replay()
    torch.cuda.synchronize()
    _check_rmsd(b, xs2, ys)
    _check_grad(b, xs2, ys)
    del g
    b.close()


def test_batched_rejects_changed_descriptors(gpu_ctx):
    from warp_md import _native as N
    from warp_md.batched import BatchedRmsd

    xs, ys = _batch([(100, 3), (200, 2)], 71)
    b = BatchedRmsd([torch.from_numpy(x).cuda() for x in xs], [torch.from_numpy(y).cuda() for y in ys])
    # gradients were not prepared
    with pytest.raises(N.WarpMdError):
        b.ctx.check(b.ctx.lib.wmd_batched_rmsd(b.ctx.handle, b._descs, b._n, 1, None))
    # a descriptor that differs from the prepared one
    b._descs[1].n_frames = 1
    with pytest.raises(N.WarpMdError):
        b.run()
    b.close()


def test_batched_rejects_host_and_misaligned_buffers():
    from warp_md import _native as N

    ctx = N.Context(0)
    x = torch.zeros(2 * 10 * 3 + 1, device="cuda")
    y = torch.zeros(10, 3, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    d = (N.BatchDesc * 1)()
    d[0].coords = x.data_ptr() + 4  # 4-byte offset: not 16-byte aligned
    d[0].ref = y.data_ptr()
    d[0].n_atoms = 10
    d[0].n_frames = 2
    d[0].rmsd = out.data_ptr()
    assert ctx.lib.wmd_batched_prepare(ctx.handle, d, 1, 0) == N.WMD_ERR_INVALID_ARG
    host = np.zeros(2)
    d[0].coords = x.data_ptr()
    d[0].rmsd = host.ctypes.data
    assert ctx.lib.wmd_batched_prepare(ctx.handle, d, 1, 0) == N.WMD_ERR_INVALID_ARG
    d[0].rmsd = out.data_ptr()
    d[0].n_atoms = -1
    assert ctx.lib.wmd_batched_prepare(ctx.handle, d, 1, 0) == N.WMD_ERR_INVALID_ARG
    ctx.close()


def test_batched_many_uneven_trajectories():
    """A scaled-down version of the 512-trajectory workload: 96 trajectories
    of 50-6000 atoms and 5-60 frames (log-uniform), all checked."""
    rng = np.random.default_rng(3)
    shapes = [(int(np.exp(rng.uniform(np.log(50), np.log(6000)))), int(rng.integers(5, 60))) for _ in range(96)]
    xs, ys = _batch(shapes, 1000)
    for layout in ("tiles", "frames", "lanes"):
        b = _run(xs, ys, with_grad=True, layout=layout)
        _check_rmsd(b, xs, ys)
        _check_grad(b, xs, ys)
        b.close()


@pytest.mark.parametrize("tile", [512, 1024])
def test_batched_lanes_tensor_maps_match_per_lane_copies(tile):
    """The lanes layout's forward reads each trajectory through its tensor map:
    frame rows when a frame is a multiple of 16 bytes, quad rows otherwise
    (the last n_frames mod 4 frames by plain loads), per-lane bulk copies for
    fewer than 4 frames.  Every lane adds its atoms in the same order either
    way, so RMSDs and gradients equal those of WARPMD_BATCHED_TMA=0 bit for
    bit, and the oracle's within the usual bars."""
    shapes = [(1000, 37), (1001, 70), (1002, 101), (1003, 66), (999, 3), (4, 33), (3, 9), (2050, 44), (2053, 35),
              (33, 64), (5, 4)]
    xs, ys = _batch(shapes, 77)
    old = os.environ.get("WARPMD_BATCHED_TMA")
    try:
        os.environ["WARPMD_BATCHED_TMA"] = "0"
        plain = _run(xs, ys, with_grad=True, tile=tile, layout="lanes")
        os.environ.pop("WARPMD_BATCHED_TMA")
        mapped = _run(xs, ys, with_grad=True, tile=tile, layout="lanes")
    finally:
        if old is None:
            os.environ.pop("WARPMD_BATCHED_TMA", None)
        else:
            os.environ["WARPMD_BATCHED_TMA"] = old
    _check_rmsd(mapped, xs, ys)
    _check_grad(mapped, xs, ys)
    for k in range(len(shapes)):
        assert torch.equal(mapped.rmsd[k], plain.rmsd[k]), k
        assert torch.equal(mapped.grads[k], plain.grads[k]), k
    plain.close()
    mapped.close()
