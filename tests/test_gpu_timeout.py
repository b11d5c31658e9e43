"""The bounded-wait error path, driven on the GPU without a fault.

Every device-side wait of the library gives up after a limit, lets the copies
it issued land, and the call reports WMD_ERR_TIMEOUT; the reference maps a CUDA
failure to an error the same way (TrajError::Unsupported,
crates/traj-gpu/src/cuda.rs:384-390) instead of hanging.  wmd_set_wait_test
shortens the consumers' limit to 2 ms and leaves the first pipeline stage of
CTA 0 unfilled, so that one wait has nothing to wait for and must run out.
Each case checks the error, then that the next call with the normal limits
returns bit-identical results to a call made before the test (the context and
the GPU stay usable).
"""
import numpy as np
import pytest

from warp_md import _native as N
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LIMIT_NS = 2_000_000


def _frames(ctx, ref_handle, fr, n_sel):
    out = np.full(fr.shape[0], -1.0, np.float64)
    rc = ctx.lib.wmd_rmsd_frames(ctx.handle, fr.data_ptr(), fr.shape[0], fr.shape[1], 3, None, n_sel, ref_handle, 1,
                                 out.ctypes.data, None)
    return rc, out


@pytest.mark.parametrize("n_atoms,n_frames", [(3001, 200), (4000, 2000)],
                         ids=["atom-major kernel", "frames-across-lanes kernel"])
def test_per_frame_wait_runs_out_and_context_recovers(n_atoms, n_frames):
    ctx = N.context(0)
    fr, ref = synth.make_trajectory(n_atoms, n_frames, 0.5, seed=71)
    x = torch.from_numpy(fr).cuda()
    r = N.Reference.from_numpy(ctx, ref)
    try:
        rc, before = _frames(ctx, r.handle, x, n_atoms)
        assert rc == N.WMD_OK, ctx.lib.wmd_last_error(ctx.handle)
        ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, LIMIT_NS, 1))
        try:
            rc, _ = _frames(ctx, r.handle, x, n_atoms)
        finally:
            ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, 0, 0))
        assert rc == N.WMD_ERR_TIMEOUT
        assert b"wait" in ctx.lib.wmd_last_error(ctx.handle)
        rc, after = _frames(ctx, r.handle, x, n_atoms)
        assert rc == N.WMD_OK, ctx.lib.wmd_last_error(ctx.handle)
        assert np.array_equal(before, after)
    finally:
        r.close()


def test_tensor_core_pairwise_wait_runs_out_and_context_recovers():
    from warp_md.plans import _PAIR_MODES

    ctx = N.context(0)
    d = synth.make_drift_trajectory(400, 300, 0.1, seed=72)
    x = torch.from_numpy(d).cuda()

    def run():
        out = np.full((d.shape[0], d.shape[0]), -1.0, np.float32)
        rc = ctx.lib.wmd_pairwise_rmsd(ctx.handle, x.data_ptr(), d.shape[0], d.shape[1], 3, None, d.shape[1],
                                       N.PAIR_RMS, _PAIR_MODES["i8x3"], out.ctypes.data, None)
        return rc, out

    rc, before = run()
    if rc == N.WMD_ERR_UNSUPPORTED:
        pytest.skip("tensor-core form not supported on this device")
    assert rc == N.WMD_OK, ctx.lib.wmd_last_error(ctx.handle)
    ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, LIMIT_NS, 1))
    try:
        rc, _ = run()
    finally:
        ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, 0, 0))
    assert rc == N.WMD_ERR_TIMEOUT
    rc, after = run()
    assert rc == N.WMD_OK, ctx.lib.wmd_last_error(ctx.handle)
    assert np.array_equal(before, after)


@pytest.mark.parametrize("entry", ["forward", "backward", "value_and_grad"])
def test_whole_frame_kernel_wait_runs_out_and_context_recovers(entry):
    """The whole-frame kernels (many small frames: wmd_rmsd_forward,
    wmd_rmsd_backward_f64, wmd_rmsd_value_and_grad) take device outputs and
    return before the GPU runs, so the timeout surfaces at the next call on
    the context, which reports it and clears it."""
    ctx = N.context(0)
    F, n = 2400, 600
    fr, ref = synth.make_trajectory(n, F, 0.5, seed=73)
    x = torch.from_numpy(fr).cuda()
    r = N.Reference.from_numpy(ctx, (ref + 0.1).astype(np.float32))
    out = torch.empty(F, dtype=torch.float64, device="cuda")
    stats = torch.empty(F, N.FRAME_STATS, dtype=torch.float64, device="cuda")
    grad = torch.empty_like(x)
    ones = torch.ones(F, dtype=torch.float64, device="cuda")

    def call():
        if entry == "forward":
            return ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, out.data_ptr(),
                                            stats.data_ptr(), None)
        if entry == "backward":
            return ctx.lib.wmd_rmsd_backward_f64(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle,
                                                 stats.data_ptr(), ones.data_ptr(), 1, grad.data_ptr(), None)
        return ctx.lib.wmd_rmsd_value_and_grad(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, None, 0,
                                               out.data_ptr(), grad.data_ptr(), None)

    try:
        ctx.check(ctx.lib.wmd_rmsd_forward(ctx.handle, x.data_ptr(), F, n, 3, None, n, r.handle, out.data_ptr(),
                                           stats.data_ptr(), None))
        assert call() == N.WMD_OK
        torch.cuda.synchronize()
        before = (out.clone(), stats.clone(), grad.clone())
        ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, LIMIT_NS, 1))
        try:
            assert call() == N.WMD_OK  # launched; the GPU has not run it yet
            torch.cuda.synchronize()
        finally:
            ctx.check(ctx.lib.wmd_set_wait_test(ctx.handle, 0, 0))
        assert call() == N.WMD_ERR_TIMEOUT
        assert call() == N.WMD_OK
        torch.cuda.synchronize()
        after = (out, stats, grad)
        for a, b in zip(before, after):
            assert torch.equal(a, b)
    finally:
        r.close()
