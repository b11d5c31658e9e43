"""Whole-frame kernels for many small frames (rmsd_vg.cu): the autograd
forward/backward that wmd_rmsd_forward / wmd_rmsd_backward run for dense
packed frames of up to 16,384 atoms and at least 16 frames per SM, and
wmd_rmsd_value_and_grad (value and gradient in one launch).

Pins: the oracle's FP64 RMSD (plan.rs:1161-1248 restated) within 1e-5 A and
its analytic FP64 gradient dRMSD/dx = (x - x_bar - R^T y_c) / (n RMSD) within
1e-5 max|g| + 1e-7 (float32 output), as for the general kernels; and the
general kernels themselves (wmd_rmsd_frames) within 1e-8 A.
"""
import numpy as np
import pytest

import oracle
from warp_md import _native as N
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ELIGIBLE = [(2400, 500), (2500, 1004), (3000, 2000)]  # frames, atoms (multiples of 4)


def _check_grad(g_gpu, g_ref):
    tol = 1e-5 * np.abs(g_ref).max() + 1e-7
    err = np.abs(g_gpu - g_ref).max()
    assert err <= tol, (err, tol)


def _traj(F, n, seed, sigma=0.3):
    fr, ref = synth.make_trajectory(n, F, sigma, seed)
    # a reference none of the frames equals: the gradient of |.| at 0 is undefined
    ref = (ref + np.random.default_rng(seed).normal(0, 0.2, ref.shape)).astype(np.float32)
    return fr, ref


@pytest.mark.parametrize("F,n", ELIGIBLE)
def test_autograd_through_whole_frame_kernels_matches_oracle(F, n):
    from warp_md.torch_ops import rmsd

    fr, ref = _traj(F, n, 11 + n)
    x = torch.from_numpy(fr).cuda().requires_grad_(True)
    val = rmsd(x, torch.from_numpy(ref).cuda())
    val.sum().backward()  # dL/drmsd: broadcast ones of stride 0
    rm, g = oracle.rmsd_grad(fr, ref)
    np.testing.assert_allclose(val.detach().cpu().numpy(), rm, rtol=0, atol=1e-5)
    _check_grad(x.grad.cpu().numpy(), g)
    # weighted upstream gradient, a contiguous float64 vector
    x.grad = None
    w = torch.linspace(-1.5, 2.0, F, device="cuda", dtype=torch.float64)
    (rmsd(x, torch.from_numpy(ref).cuda()) * w).sum().backward()
    _check_grad(x.grad.cpu().numpy(), g * w.cpu().numpy()[:, None, None])


def test_value_and_grad_matches_oracle_with_strided_and_broadcast_weights():
    from warp_md.torch_ops import rmsd_value_and_grad

    F, n = 2400, 604
    fr, ref = _traj(F, n, 5)
    x = torch.from_numpy(fr).cuda()
    y = torch.from_numpy(ref).cuda()
    rm, g = oracle.rmsd_grad(fr, ref)
    val, grad = rmsd_value_and_grad(x, y)
    np.testing.assert_allclose(val.cpu().numpy(), rm, rtol=0, atol=1e-5)
    _check_grad(grad.cpu().numpy(), g)
    # every other element of a longer vector (stride 2), with zeros and signs
    wl = torch.randn(2 * F, device="cuda", dtype=torch.float64)
    wl[0:200:2] = 0.0
    w = wl[::2]
    assert w.stride(0) == 2
    val, grad = rmsd_value_and_grad(x, y, w)
    np.testing.assert_allclose(val.cpu().numpy(), rm, rtol=0, atol=1e-5)
    _check_grad(grad.cpu().numpy(), g * w.cpu().numpy()[:, None, None])
    # one weight for every frame (stride 0)
    w0 = torch.tensor(2.5, device="cuda", dtype=torch.float64).expand(F)
    assert w0.stride(0) == 0
    _, grad = rmsd_value_and_grad(x, y, w0)
    _check_grad(grad.cpu().numpy(), 2.5 * g)


def test_value_and_grad_general_shapes_take_the_two_kernel_route():
    """Too few frames, an atom count that is not a multiple of 4, and an index
    selection: forward + backward of the general kernels, same results."""
    from warp_md.torch_ops import rmsd_value_and_grad

    for F, n, sel in [(100, 800, None), (2400, 501, None), (2400, 900, np.arange(0, 900, 3))]:
        fr, _ = synth.make_trajectory(n, F, 0.3, 21)
        s = None if sel is None else sel
        ref = fr[0] if s is None else fr[0][s]
        ref = (ref + np.random.default_rng(3).normal(0, 0.2, ref.shape)).astype(np.float32)
        x = torch.from_numpy(fr).cuda()
        ts = None if s is None else torch.from_numpy(s.astype(np.int32)).cuda()
        w = torch.linspace(0.5, 1.5, F, device="cuda", dtype=torch.float64)
        val, grad = rmsd_value_and_grad(x, torch.from_numpy(ref).cuda(), w, ts)
        rm, g = oracle.rmsd_grad(fr, ref, selection=s)
        np.testing.assert_allclose(val.cpu().numpy(), rm, rtol=0, atol=1e-5)
        _check_grad(grad.cpu().numpy(), g * w.cpu().numpy()[:, None, None])


def test_whole_frame_forward_agrees_with_general_kernels_and_refines_near_zero_frames():
    """wmd_rmsd_forward (whole-frame kernel) against wmd_rmsd_frames (the
    frames-across-lanes kernel and its finisher) on the same frames, some of
    them copies of the reference or within 1e-5 A of it (explicit residuals)."""
    ctx = N.context(0)
    F, n = 2400, 1000
    fr, ref = synth.make_trajectory(n, F, (0.05, 3.0), 31)
    fr[7] = ref
    fr[2399] = ref
    rng = np.random.default_rng(2)
    fr[100] = (ref + rng.normal(0, 1e-5, ref.shape)).astype(np.float32)
    x = torch.from_numpy(fr).cuda()
    r = N.Reference.from_numpy(ctx, ref)
    try:
        out = torch.empty(F, dtype=torch.float64, device="cuda")
        stats = torch.empty(F, N.FRAME_STATS, dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, out.data_ptr(),
                                           stats.data_ptr(), None))
        general = torch.empty(F, dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, 1,
                                          general.data_ptr(), None))
        torch.cuda.synchronize()
        got, exp = out.cpu().numpy(), general.cpu().numpy()
        np.testing.assert_allclose(got, exp, rtol=0, atol=1e-8)
        np.testing.assert_array_equal(stats[:, 13].cpu().numpy(), got)
        assert got[7] < 1e-9 and got[2399] < 1e-9
        _, o64 = oracle.rmsd_frames(fr[[100]], ref)
        assert abs(got[100] - o64[0]) < 1e-8
    finally:
        r.close()


def test_value_and_grad_is_reproducible():
    from warp_md.torch_ops import rmsd_value_and_grad

    fr, ref = _traj(2400, 800, 41)
    x = torch.from_numpy(fr).cuda()
    y = torch.from_numpy(ref).cuda()
    v1, g1 = rmsd_value_and_grad(x, y)
    v2, g2 = rmsd_value_and_grad(x, y)
    assert torch.equal(v1, v2) and torch.equal(g1, g2)


def test_whole_frame_kernels_from_a_fresh_thread():
    """The whole-frame kernels encode their tensor maps through the driver
    API, which needs the device's context current on the calling thread; a
    thread that made no CUDA call yet (the autograd engine's workers, a user's
    thread) must work as the main thread does."""
    import threading

    from warp_md.torch_ops import rmsd_value_and_grad

    fr, ref = _traj(2400, 400, 51)
    x = torch.from_numpy(fr).cuda()
    y = torch.from_numpy(ref).cuda()
    main_v, main_g = rmsd_value_and_grad(x, y)
    torch.cuda.synchronize()
    box = {}

    def work():
        try:
            v, g = rmsd_value_and_grad(x, y)
            torch.cuda.synchronize()
            box["v"], box["g"] = v.cpu(), g.cpu()
        except Exception as exc:  # reported below
            box["err"] = exc

    t = threading.Thread(target=work)
    t.start()
    t.join(timeout=120)
    assert "err" not in box, box.get("err")
    assert torch.equal(box["v"], main_v.cpu()) and torch.equal(box["g"], main_g.cpu())
