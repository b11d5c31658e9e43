"""Fluctuations (wmd_rmsf: RmsfPlan, AtomicFluctPlan, BfactorsPlan,
AtomicAdpPlan, the fluct wrappers) and per-residue RMSD (wmd_rmsd_per_group:
RmsdPerResPlan) on the GPU against the oracle.

Tolerances: RMSF within 2e-6 relative + 1e-6 A and ADP within 4e-6 relative
+ 1e-6 A^2 of the oracle's FP64 values (the outputs are float32);
per-residue RMSD within 1e-5 A, the per-frame RMSD bar.
"""
import numpy as np
import pytest

import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _rmsf(coords, sel=None, n_sel=None, stride=3, device_io=False):
    from warp_md import _native as N

    ctx = N.context(0)
    n = sel.size if sel is not None else (coords.shape[1] if n_sel is None else n_sel)
    sel_arr = None if sel is None else np.ascontiguousarray(sel, np.uint32)
    if device_io:
        x = torch.from_numpy(np.ascontiguousarray(coords)).cuda()
        r = torch.empty(n, device="cuda")
        a = torch.empty(n, 6, device="cuda")
        s = None if sel_arr is None else torch.from_numpy(sel_arr.astype(np.int32)).cuda()
        ctx.check(ctx.lib.wmd_rmsf(ctx.handle, x.data_ptr(), coords.shape[0], coords.shape[1], stride,
                                   None if s is None else s.data_ptr(), n, r.data_ptr(), a.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        return r.cpu().numpy(), a.cpu().numpy()
    r = np.empty(n, np.float32)
    a = np.empty((n, 6), np.float32)
    c = np.ascontiguousarray(coords, np.float32)
    ctx.check(ctx.lib.wmd_rmsf(ctx.handle, c.ctypes.data, c.shape[0], c.shape[1], stride, N.ptr(sel_arr), n,
                               r.ctypes.data, a.ctypes.data, None))
    return r, a


def _check(r, a, orr, oa):
    assert np.all(np.abs(r - orr) <= 2e-6 * np.abs(orr) + 1e-6), np.abs(r - orr).max()
    assert np.all(np.abs(a - oa) <= 4e-6 * np.abs(oa).max() + 1e-6), np.abs(a - oa).max()


@pytest.mark.parametrize("device_io", [False, True])
def test_rmsf_dense_and_selection_match_oracle(device_io):
    fr, _ = synth.make_trajectory(3001, 257, (0.05, 3.0), 4)
    r, a = _rmsf(fr, device_io=device_io)
    orr, oa = oracle.rmsf(fr)
    _check(r, a, orr, oa)
    sel = np.sort(np.random.default_rng(0).choice(3001, 700, replace=False)).astype(np.uint32)
    r, a = _rmsf(fr, sel=sel, device_io=device_io)
    orr, oa = oracle.rmsf(fr, selection=sel)
    _check(r, a, orr, oa)


def test_rmsf_stride4_edges_and_host_chunks():
    fr, _ = synth.make_trajectory(50, 9, 0.5, 5)
    fr4 = np.concatenate([fr, np.ones(fr.shape[:2] + (1,), np.float32)], axis=2)
    r, a = _rmsf(fr4, stride=4)
    orr, oa = oracle.rmsf(fr4)
    _check(r, a, orr, oa)
    # one frame: zero fluctuation; a constant atom; far-from-origin coordinates
    r, a = _rmsf(fr[:1])
    np.testing.assert_array_equal(r, 0.0)
    big = fr.copy() + np.float32(5000.0)
    big[:, 3] = big[0, 3]
    r, a = _rmsf(big)
    orr, oa = oracle.rmsf(big)
    _check(r, a, orr, oa)
    assert r[3] == 0.0
    # 100,000 atoms x 700 frames through host chunks (840 MB > one chunk buffer)
    x, _ = synth.make_trajectory_torch(100_000, 700, (0.05, 3.0), seed=7, device="cuda")
    host = x.cpu().numpy()
    sel = np.arange(0, 100_000, 97, dtype=np.uint32)
    r, a = _rmsf(host, sel=sel)
    orr, oa = oracle.rmsf(host, selection=sel)
    _check(r, a, orr, oa)


def test_fluct_plans_and_wrappers_reference_known_answers():
    import warp_md
    from warp_md.analysis.fluct import atomicfluct, bfactors, rmsf
    from warp_md.analysis.trajectory import ArrayTrajectory

    coords = np.zeros((3, 4, 3), dtype=np.float32)
    coords[:, 1, 0] = [0.0, 1.0, 2.0]
    coords[:, 3, 0] = [2.0, 3.0, 4.0]
    table = {"name": ["CA", "CB", "CA", "CB"], "resname": ["ALA", "ALA", "GLY", "GLY"], "resid": [1, 1, 2, 2],
             "chain_id": [0, 0, 0, 0], "mass": [1.0, 1.0, 1.0, 1.0]}
    system = warp_md.System.from_arrays(table, positions0=coords[0])
    r0 = np.sqrt(2.0 / 3.0)
    # test_rmsf_byatom_byres
    data = rmsf(ArrayTrajectory(coords), system, mask="resid 1:2", byres=False)
    assert data.shape == (4, 2)
    np.testing.assert_allclose(data[:, 1], [0.0, r0, 0.0, r0], rtol=1e-6)
    byres = rmsf(ArrayTrajectory(coords), system, mask="resid 1:2", byres=True)
    np.testing.assert_allclose(byres, [[1.0, r0 / 2.0], [2.0, r0 / 2.0]], rtol=1e-6)
    # test_bfactors_bymask
    data = bfactors(ArrayTrajectory(coords), system, mask="resid 1:2", byres=False, bymask=True)
    np.testing.assert_allclose(data[0, 1], 8.0 * np.pi * np.pi / 3.0 * r0 * r0 * 0.5, rtol=1e-6)
    # test_atomicfluct_calcadp
    data = atomicfluct(ArrayTrajectory(coords), system, mask="resid 1:2", calcadp=True)
    assert data.shape == (4, 7)
    np.testing.assert_allclose(data[[1, 3], 1], [2.0 / 3.0, 2.0 / 3.0], rtol=1e-6)
    np.testing.assert_allclose(data[:, 2:], 0.0, atol=1e-6)
    # frame subsets [2, 0] (test_rmsf_native_frame_indices..., test_atomicfluct_adp_native...)
    traj = warp_md.Trajectory.from_numpy(coords)
    data = rmsf(traj, system, mask="resid 1:2", frame_indices=[2, 0], chunk_frames=1)
    np.testing.assert_allclose(data[:, 1], [0.0, 1.0, 0.0, 1.0], rtol=1e-6)
    data = atomicfluct(traj, system, mask="resid 1:2", calcadp=True, frame_indices=[2, 0])
    np.testing.assert_allclose(data[[1, 3], 1], [1.0, 1.0], rtol=1e-6)
    # the plan classes
    sel = system.select("all")
    np.testing.assert_allclose(warp_md.RmsfPlan(sel).run(traj, system), [0.0, r0, 0.0, r0], rtol=1e-6)
    np.testing.assert_allclose(warp_md.AtomicFluctPlan(sel).run(traj, system), [0.0, r0, 0.0, r0], rtol=1e-6)
    np.testing.assert_allclose(warp_md.BfactorsPlan(sel).run(traj, system),
                               8.0 * np.pi * np.pi / 3.0 * np.array([0.0, r0, 0.0, r0]) ** 2, rtol=1e-6)
    adp = warp_md.AtomicAdpPlan(sel).run(traj, system)
    assert adp.shape == (4, 6)
    np.testing.assert_allclose(adp[[1, 3], 0], [2.0 / 3.0, 2.0 / 3.0], rtol=1e-6)
    assert warp_md.AtomicAdpPlan(sel).run(warp_md.Trajectory.from_numpy(coords[:0]), system).shape == (0, 6)


def test_rmsd_per_residue_matches_oracle():
    import warp_md

    n = 1200
    fr, ref = synth.make_trajectory(n, 11, 0.6, 14)
    resid = (np.arange(n) // 9 + 1).astype(np.int64)
    table = {"name": ["CA" if i % 9 == 1 else "X" for i in range(n)], "resid": resid}
    system = warp_md.System.from_arrays(table, positions0=ref)
    traj = warp_md.Trajectory.from_numpy(fr)
    for expr in ("all", "name CA", "resid 5:40"):
        sel = system.select(expr)
        idx = sel.as_array()
        order = np.unique(resid[idx])
        groups = [idx[resid[idx] == r] for r in order]
        for mode, ref_all in (("topology", ref), ("frame0", fr[0])):
            for align in (True, False):
                rids, got = warp_md.RmsdPerResPlan(sel, reference=mode, align=align).run(traj, system)
                np.testing.assert_array_equal(rids, order.astype(np.int32))
                want = oracle.rmsd_perres(fr, ref_all, groups, selection=idx, align=align)
                assert got.shape == want.shape and got.dtype == np.float32
                np.testing.assert_allclose(got, want, rtol=0, atol=1e-5, err_msg=f"{expr} {mode} {align}")


def test_group_ref_validates_groups():
    from warp_md import _native as N

    ctx = N.context(0)
    _, ref = synth.make_trajectory(20, 2, 0.5, 3)
    goff = np.array([0, 3, 5], np.uint32)
    bad = np.array([0, 1, 2, 3, 20], np.uint32)  # 20 is out of range
    with pytest.raises(N.WarpMdError):
        N.GroupRef(ctx, ref, goff, bad)
    with pytest.raises(N.WarpMdError):
        N.GroupRef(ctx, ref, np.array([0, 3, 2], np.uint32), bad[:3])


@pytest.mark.parametrize("stride", [3, 4])
def test_rmsd_per_group_many_frames_and_group_shapes(stride):
    """wmd_rmsd_per_group with superposition, groups that are not one run of
    consecutive atoms (the item kernel): 300 frames of 6,000 atoms, every
    10th atom aligned (a device selection),
    groups covering every atom -- ten-atom runs, one group of 2,500 atoms
    (larger than a 2,048-position tile) and one scattered group -- against
    the oracle's RmsdPerResPlan restatement (rms.rs:431-686) within 1e-5 A."""
    from warp_md import _native as N

    ctx = N.context(0)
    n, F = 6000, 300
    fr, ref = synth.make_trajectory(n, F, (0.1, 2.0), 23)
    fr[5] = ref
    sel = np.arange(0, n, 10, dtype=np.uint32)
    scattered = np.arange(3, n, 97)
    rest = np.setdiff1d(np.arange(2500, n), scattered)
    groups = [np.arange(0, 2500)] + [rest[i:i + 10] for i in range(0, rest.size, 10)] + [scattered]
    goff = np.zeros(len(groups) + 1, np.uint32)
    goff[1:] = np.cumsum([g.size for g in groups])
    gat = np.concatenate(groups).astype(np.uint32)
    data = fr if stride == 3 else np.concatenate([fr, np.ones(fr.shape[:2] + (1,), np.float32)], axis=2)
    x = torch.from_numpy(np.ascontiguousarray(data)).cuda()
    rr = N.Reference.from_numpy(ctx, ref[sel])
    gref = N.GroupRef(ctx, ref, goff, gat)
    dsel = torch.from_numpy(sel.astype(np.int32)).cuda()
    out = torch.empty(F, len(groups), device="cuda")
    try:
        ctx.check(ctx.lib.wmd_rmsd_per_group(ctx.handle, x.data_ptr(), F, n, stride, dsel.data_ptr(), sel.size,
                                             rr.handle, gref.handle, 1, out.data_ptr(), None))
        torch.cuda.synchronize()
        want = oracle.rmsd_perres(fr, ref, groups, selection=sel, align=True)
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-5)
        assert np.abs(got[5]).max() < 1e-5  # the frame equal to the reference
    finally:
        gref.close()
        rr.close()


@pytest.mark.parametrize("stride", [3, 4])
def test_rmsd_per_group_contiguous_groups_edges(stride):
    """Groups that cover consecutive atoms (no index load per position):
    residues of 1 to 30 atoms, empty groups, one group of 2,100 atoms (larger
    than a 2,048-position block, walked in tiles), an odd atom count and a frame
    base 4 bytes off 16-byte alignment, with and without superposition, against
    the oracle within 1e-5 A + 1.2e-7 relative (one float32 ulp: values reach
    ~260 A without superposition)."""
    from warp_md import _native as N

    ctx = N.context(0)
    n, F = 7001, 257
    fr, ref = synth.make_trajectory(n, F, (0.1, 2.0), 29)
    fr[3] = ref
    rng = np.random.default_rng(4)
    sizes, left = [], n
    while left > 0:
        k = 2100 if len(sizes) == 40 else (0 if len(sizes) % 17 == 5 else int(rng.integers(1, 31)))
        k = min(k, left)
        sizes.append(k)
        left -= k
    goff = np.zeros(len(sizes) + 1, np.uint32)
    goff[1:] = np.cumsum(sizes)
    assert goff[-1] == n and 2100 in sizes and 0 in sizes
    groups = [np.arange(goff[i], goff[i + 1]) for i in range(len(sizes))]
    data = fr if stride == 3 else np.concatenate([fr, np.ones(fr.shape[:2] + (1,), np.float32)], axis=2)
    flat = torch.zeros(data.size + 1, device="cuda")
    flat[1:] = torch.from_numpy(np.ascontiguousarray(data)).reshape(-1).cuda()
    x = flat[1:]
    assert x.data_ptr() % 16 == 4
    sel = np.arange(0, n, 7, dtype=np.uint32)
    rr = N.Reference.from_numpy(ctx, ref[sel])
    gref = N.GroupRef(ctx, ref, goff, np.arange(n, dtype=np.uint32))
    dsel = torch.from_numpy(sel.astype(np.int32)).cuda()
    try:
        for align in (1, 0):
            out = torch.full((F, len(sizes)), -1.0, device="cuda")
            ctx.check(ctx.lib.wmd_rmsd_per_group(ctx.handle, x.data_ptr(), F, n, stride, dsel.data_ptr(), sel.size,
                                                 rr.handle, gref.handle, align, out.data_ptr(), None))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            want = oracle.rmsd_perres(fr, ref, groups, selection=sel, align=bool(align))
            np.testing.assert_allclose(got, want, rtol=1.2e-7, atol=1e-5, err_msg=str(align))
            assert np.all(got[:, np.array(sizes) == 0] == 0.0)
            if align:
                assert np.abs(got[3]).max() < 1e-5
    finally:
        gref.close()
        rr.close()
