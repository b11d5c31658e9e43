"""wmd_rmsd_frames_noalloc: the per-frame RMSD entry point for callers that
cannot allocate (no context, no reference object, scratch in a fixed array
inside the library).  Checked through the C ABI against wmd_rmsd_frames on
the same inputs, for two calls in a row with different shapes (the second must
not see the first call's leftovers in the shared scratch array), within the
per-frame tolerance of 1e-5 A.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from warp_md import _native as N
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def _existing(ctx, coords, ref, n_sel=None):
    """wmd_rmsd_frames over the first n_sel atoms of each frame (an explicit
    index list when n_sel < n_atoms, as that entry point asks)."""
    n_sel = ref.shape[0] if n_sel is None else n_sel
    r = N.Reference(ctx, ref.data_ptr(), n_sel, ref.shape[1], keepalive=ref)
    out = torch.empty(coords.shape[0], dtype=torch.float64, device="cuda")
    sel = None
    if n_sel < coords.shape[1]:
        sel = torch.arange(n_sel, dtype=torch.int32, device="cuda")
    ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, coords.data_ptr(), coords.shape[0], coords.shape[1],
                                      coords.shape[2], None if sel is None else sel.data_ptr(), n_sel, r.handle, 1,
                                      out.data_ptr(), None))
    torch.cuda.synchronize()
    r.close()
    return out.cpu().numpy()


def _noalloc(lib, coords, ref, n_sel=None):
    n_sel = ref.shape[0] if n_sel is None else n_sel
    out = torch.full((coords.shape[0],), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.wmd_rmsd_frames_noalloc(coords.data_ptr(), coords.shape[0], coords.shape[1], coords.shape[2],
                                     ref.data_ptr(), n_sel, ref.shape[1], out.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _xyzw(a):
    return np.concatenate([a, np.full(a.shape[:-1] + (1,), 7.0, np.float32)], axis=-1)


def test_noalloc_matches_existing_entry_point_twice():
    ctx = N.context(0)
    lib = ctx.lib
    # first call: 3,000 atoms x 300 frames (three tiles per frame)
    fr, ref = synth.make_trajectory(3000, 300, (0.05, 3.0), seed=41)
    x = torch.from_numpy(fr).cuda()
    y = torch.from_numpy(ref).cuda()
    rc, got = _noalloc(lib, x, y)
    assert rc == N.WMD_OK, lib.wmd_last_error(None)
    np.testing.assert_allclose(got, _existing(ctx, x, y), rtol=0, atol=TOL)
    # second call: a different shape, the largest selection accepted, and one
    # frame equal to the reference (the explicit residual pass)
    fr2, ref2 = synth.make_trajectory(65536, 40, 0.5, seed=42)
    fr2[7] = ref2
    x2 = torch.from_numpy(fr2).cuda()
    y2 = torch.from_numpy(ref2).cuda()
    rc, got2 = _noalloc(lib, x2, y2)
    assert rc == N.WMD_OK, lib.wmd_last_error(None)
    np.testing.assert_allclose(got2, _existing(ctx, x2, y2), rtol=0, atol=TOL)
    assert got2[7] < 1e-9


def test_noalloc_rejects_selections_beyond_its_scratch():
    lib = N.load()
    x = torch.zeros((2, 65537, 3), dtype=torch.float32, device="cuda")
    rc, _ = _noalloc(lib, x, x[0])
    assert rc == N.WMD_ERR_INVALID_ARG
    assert b"65536" in lib.wmd_last_error(None)


def test_noalloc_several_batches_odd_atoms_strides_and_prefix_selection():
    """Shapes beyond a single launch of the fixed scratch: 1,001 atoms (frames
    not a multiple of 16 bytes) over 60,000 frames, which the 16 MiB array
    splits into two batches; xyzw frames and reference; and a selection of the
    first atoms of larger frames."""
    ctx = N.context(0)
    lib = ctx.lib
    # two batches: 1,001 atoms need one tile, 256 bytes of scratch per frame
    fr, ref = synth.make_trajectory(1001, 60000, (0.05, 3.0), seed=43)
    fr[59999] = ref
    x = torch.from_numpy(fr).cuda()
    y = torch.from_numpy(ref).cuda()
    rc, got = _noalloc(lib, x, y)
    assert rc == N.WMD_OK, lib.wmd_last_error(None)
    np.testing.assert_allclose(got, _existing(ctx, x, y), rtol=0, atol=TOL)
    assert got[59999] < 1e-9
    del x
    # stride 4 frames and reference
    fr4, ref4 = synth.make_trajectory(2500, 90, 0.7, seed=44)
    x4 = torch.from_numpy(_xyzw(fr4)).cuda()
    y4 = torch.from_numpy(_xyzw(ref4)).cuda()
    rc, got4 = _noalloc(lib, x4, y4)
    assert rc == N.WMD_OK, lib.wmd_last_error(None)
    np.testing.assert_allclose(got4, _existing(ctx, x4, y4), rtol=0, atol=TOL)
    # the first 1,700 of 2,500 atoms, frames starting 4 bytes past a 16-byte
    # boundary (the kernels must not bulk-copy from such a base)
    buf = torch.empty(fr4.size + 1, dtype=torch.float32, device="cuda")
    xs = buf[1:].view(fr4.shape)
    xs.copy_(torch.from_numpy(fr4))
    assert xs.data_ptr() % 16 == 4
    ys = torch.from_numpy(ref4[:1700].copy()).cuda()
    rc, gots = _noalloc(lib, xs, ys, 1700)
    assert rc == N.WMD_OK, lib.wmd_last_error(None)
    np.testing.assert_allclose(gots, _existing(ctx, xs, ys, 1700), rtol=0, atol=TOL)


def test_noalloc_rejects_another_devices_or_host_memory():
    lib = N.load()
    x = np.zeros((2, 10, 3), np.float32)
    out = np.zeros(2, np.float64)
    rc = lib.wmd_rmsd_frames_noalloc(x.ctypes.data, 2, 10, 3, x.ctypes.data, 10, 3, out.ctypes.data, None)
    assert rc == N.WMD_ERR_INVALID_ARG
    assert b"device memory" in lib.wmd_last_error(None)
