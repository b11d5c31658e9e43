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


def _existing(ctx, coords, ref):
    r = N.Reference(ctx, ref.data_ptr(), ref.shape[0], 3, keepalive=ref)
    out = torch.empty(coords.shape[0], dtype=torch.float64, device="cuda")
    ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, coords.data_ptr(), coords.shape[0], coords.shape[1], 3, None,
                                      ref.shape[0], r.handle, 1, out.data_ptr(), None))
    torch.cuda.synchronize()
    r.close()
    return out.cpu().numpy()


def _noalloc(lib, coords, ref, n_sel=None):
    n_sel = ref.shape[0] if n_sel is None else n_sel
    out = torch.full((coords.shape[0],), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.wmd_rmsd_frames_noalloc(coords.data_ptr(), coords.shape[0], coords.shape[1], 3, ref.data_ptr(), n_sel,
                                     3, out.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


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
