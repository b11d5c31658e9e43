"""Per-frame RMSD on the GPU (through the C ABI) against the CPU oracle.

Tolerance: 1e-5 A on the FP64 result for every case (the target for per-frame
RMSD); float32 outputs of the Plan API are compared to the oracle's float32
results with the same bound.
"""
import ctypes

import numpy as np
import pytest

import oracle
import warp_md
from warp_md import _native as N
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def gpu_rmsd(ctx, coords, ref, sel=None, align=True, stride=3, device_io=False):
    """Calls wmd_rmsd_frames with host numpy (default) or device tensors."""
    c = np.ascontiguousarray(coords, np.float32)
    if stride == 4 and c.shape[2] == 3:
        c = np.concatenate([c, np.ones(c.shape[:2] + (1,), np.float32)], axis=2)
    r = N.Reference.from_numpy(ctx, ref)
    F, n_atoms = c.shape[0], c.shape[1]
    n_sel = r.n_sel
    try:
        if device_io:
            dc = torch.from_numpy(c).cuda()
            dout = torch.empty(F, dtype=torch.float64, device="cuda")
            dsel = None if sel is None else torch.from_numpy(np.asarray(sel, np.int32)).cuda()
            ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, dc.data_ptr(), F, n_atoms, stride,
                                              None if dsel is None else dsel.data_ptr(), n_sel, r.handle,
                                              int(align), dout.data_ptr(), None))
            torch.cuda.synchronize()
            return dout.cpu().numpy()
        out = np.empty(F, np.float64)
        s = None if sel is None else np.ascontiguousarray(sel, np.uint32)
        ctx.check(ctx.lib.wmd_rmsd_frames(ctx.handle, c.ctypes.data, F, n_atoms, stride, N.ptr(s), n_sel, r.handle,
                                          int(align), out.ctypes.data, None))
        return out
    finally:
        r.close()


def test_golden_cases(gpu_ctx, golden):
    for name in sorted(k[7:] for k in golden.files if k.startswith("frames_")):
        fr, ref = golden["frames_" + name], golden["ref_" + name]
        got = gpu_rmsd(gpu_ctx, fr, ref)
        np.testing.assert_allclose(got, golden["expect_aligned_" + name], rtol=0, atol=TOL, err_msg=name)
        raw = gpu_rmsd(gpu_ctx, fr, ref, align=False)
        np.testing.assert_allclose(raw, golden["expect_raw_" + name], rtol=0, atol=TOL, err_msg=name)


def test_plain_per_frame_workload(gpu_ctx):
    # 3,000-atom selection, 1,000 frames, sigma = 0.5 A, reference = frame 0
    fr, _ = synth.make_trajectory(3000, 1000, 0.5, seed=0)
    ref = fr[0].copy()
    got = gpu_rmsd(gpu_ctx, fr, ref)
    _, exp = oracle.rmsd_frames(fr, ref)
    err = np.abs(got - exp)
    assert err.max() < TOL, err.max()
    assert got[0] < TOL


@pytest.mark.parametrize("n_atoms", [1, 2, 3, 31, 33, 255, 1023, 1024, 1025, 2049, 4097])
@pytest.mark.parametrize("n_frames", [1, 2, 127])
def test_odd_shapes(gpu_ctx, n_atoms, n_frames):
    fr, ref = synth.make_trajectory(n_atoms, n_frames, 0.3, seed=n_atoms * 7 + n_frames)
    got = gpu_rmsd(gpu_ctx, fr, ref)
    _, exp = oracle.rmsd_frames(fr, ref)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)


@pytest.mark.parametrize("n_atoms,n_frames,stride", [
    (4, 1, 3), (36, 31, 3), (100, 33, 3), (2052, 65, 3), (4100, 3, 3), (8192, 40, 3),
    (999, 33, 4), (2049, 5, 4), (64, 300, 4)])
def test_frames_across_lanes_shapes(gpu_ctx, n_atoms, n_frames, stride):
    """Shapes the frames-across-lanes kernel takes (packed xyz with n_atoms % 4
    == 0, or xyzw): partial last stages and tiles, frame groups that are not
    multiples of 32, both metrics."""
    fr, ref = synth.make_trajectory(n_atoms, n_frames, (0.05, 2.0), seed=n_atoms + 31 * n_frames)
    got = gpu_rmsd(gpu_ctx, fr, ref, stride=stride, device_io=True)
    _, exp = oracle.rmsd_frames(fr, ref)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
    raw = gpu_rmsd(gpu_ctx, fr, ref, stride=stride, align=False, device_io=True)
    _, expr = oracle.rmsd_frames(fr, ref, align=False)
    np.testing.assert_allclose(raw, expr, rtol=0, atol=TOL)
    # a dense prefix of the frame (n_sel < n_atoms)
    k = max(1, n_atoms // 2)
    got = gpu_rmsd(gpu_ctx, fr, ref[:k], stride=stride, device_io=True)
    _, exp = oracle.rmsd_frames(fr, ref[:k], selection=np.arange(k))
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)


@pytest.mark.parametrize("stride", [3, 4])
@pytest.mark.parametrize("device_io", [False, True])
def test_layouts_and_memory_kinds(gpu_ctx, stride, device_io):
    fr, ref = synth.make_trajectory(2500, 37, (0.05, 3.0), seed=5)
    got = gpu_rmsd(gpu_ctx, fr, ref, stride=stride, device_io=device_io)
    _, exp = oracle.rmsd_frames(fr, ref)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)


@pytest.mark.parametrize("device_io", [False, True])
def test_selection_gather(gpu_ctx, device_io):
    rng = np.random.default_rng(2)
    fr, _ = synth.make_trajectory(3000, 20, 0.5, seed=9)
    sel = np.sort(rng.choice(3000, 1500, replace=False)).astype(np.uint32)
    ref = fr[3][sel]
    got = gpu_rmsd(gpu_ctx, fr, ref, sel=sel, device_io=device_io)
    _, exp = oracle.rmsd_frames(fr, ref, selection=sel)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
    raw = gpu_rmsd(gpu_ctx, fr, ref, sel=sel, align=False, device_io=device_io)
    _, expr = oracle.rmsd_frames(fr, ref, selection=sel, align=False)
    np.testing.assert_allclose(raw, expr, rtol=0, atol=TOL)


@pytest.mark.parametrize("step,offset,n_atoms", [(2, 3, 20000), (3, 0, 4000), (1, 7, 3000), (4, 5, 2500),
                                                 (10, 1, 3000)])
def test_sorted_sparse_selection_spans(gpu_ctx, step, offset, n_atoms):
    """Sorted host selections (every step-th atom from an offset) at least 1/4
    dense run as the atom span they cover with zero-weight gaps
    (frames-across-lanes kernel); sparser ones and an unsorted copy of the
    same selection take the gathered path; all match the oracle, aligned and
    raw."""
    fr, _ = synth.make_trajectory(n_atoms, 70, (0.05, 2.0), seed=step * 100 + offset)
    sel = np.arange(offset, n_atoms, step, dtype=np.uint32)
    ref = fr[5][sel]
    for s in (sel, sel[::-1].copy()):
        r = fr[5][s]
        got = gpu_rmsd(gpu_ctx, fr, r, sel=s)
        _, exp = oracle.rmsd_frames(fr, r, selection=s)
        np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
        raw = gpu_rmsd(gpu_ctx, fr, r, sel=s, align=False)
        _, expr = oracle.rmsd_frames(fr, r, selection=s, align=False)
        np.testing.assert_allclose(raw, expr, rtol=0, atol=TOL)
    assert ref.shape[0] == sel.size


def test_unaligned_device_base(gpu_ctx):
    fr, ref = synth.make_trajectory(777, 9, 0.4, seed=12)
    flat = torch.empty(fr.size + 1, dtype=torch.float32, device="cuda")
    flat[1:] = torch.from_numpy(fr.reshape(-1)).cuda()
    view = flat[1:]  # base pointer 4 bytes past a 16-byte boundary
    assert view.data_ptr() % 16 != 0
    r = N.Reference.from_numpy(gpu_ctx, ref)
    out = torch.empty(9, dtype=torch.float64, device="cuda")
    gpu_ctx.check(gpu_ctx.lib.wmd_rmsd_frames(gpu_ctx.handle, view.data_ptr(), 9, 777, 3, None, 777, r.handle, 1,
                                              out.data_ptr(), None))
    torch.cuda.synchronize()
    _, exp = oracle.rmsd_frames(fr, ref)
    np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=0, atol=TOL)
    r.close()


def test_bitwise_deterministic(gpu_ctx):
    fr, ref = synth.make_trajectory(5000, 64, 0.5, seed=21)
    a = gpu_rmsd(gpu_ctx, fr, ref, device_io=True)
    b = gpu_rmsd(gpu_ctx, fr, ref, device_io=True)
    np.testing.assert_array_equal(a, b)
    c = gpu_rmsd(gpu_ctx, fr, ref)  # chunked host path, same per-frame arithmetic
    np.testing.assert_array_equal(a, c)


def test_identical_and_empty(gpu_ctx):
    fr, ref = synth.make_trajectory(100, 3, 0.0, seed=1)
    same = np.stack([ref, ref, ref])
    assert np.all(gpu_rmsd(gpu_ctx, same, ref) < 1e-9)  # explicit residual pass near zero
    big, bref = synth.make_trajectory(20000, 4, 0.5, seed=2)
    big[2] = bref  # one frame equal to the reference, among ordinary frames
    got = gpu_rmsd(gpu_ctx, big, bref)
    _, exp = oracle.rmsd_frames(big, bref)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
    assert got[2] < 1e-9
    out = gpu_rmsd(gpu_ctx, fr, np.zeros((0, 3), np.float32), sel=np.zeros(0, np.uint32))
    assert np.all(out == 0)


def test_errors(gpu_ctx):
    fr, ref = synth.make_trajectory(10, 2, 0.1, seed=3)
    r = N.Reference.from_numpy(gpu_ctx, ref)
    out = np.empty(2)
    rc = gpu_ctx.lib.wmd_rmsd_frames(gpu_ctx.handle, fr.ctypes.data, 2, 10, 3, None, 9, r.handle, 1,
                                     out.ctypes.data, None)
    assert rc == N.WMD_ERR_MISMATCH
    rc = gpu_ctx.lib.wmd_rmsd_frames(gpu_ctx.handle, fr.ctypes.data, 2, 10, 5, None, 10, r.handle, 1,
                                     out.ctypes.data, None)
    assert rc == N.WMD_ERR_INVALID_ARG
    bad = np.arange(10, dtype=np.uint32)
    bad[3] = 10
    rc = gpu_ctx.lib.wmd_rmsd_frames(gpu_ctx.handle, fr.ctypes.data, 2, 10, 3, bad.ctypes.data, 10, r.handle, 1,
                                     out.ctypes.data, None)
    assert rc == N.WMD_ERR_INVALID_ARG
    assert b"out of range" in gpu_ctx.lib.wmd_last_error(gpu_ctx.handle)
    r.close()


def test_covariance_dropin(gpu_ctx):
    fr, ref = synth.make_trajectory(1500, 8, 0.5, seed=4)
    r = N.Reference.from_numpy(gpu_ctx, ref)
    cov = np.empty((8, 9), np.float32)
    x2 = np.empty(8, np.float32)
    y2 = np.empty(8, np.float32)
    gpu_ctx.check(gpu_ctx.lib.wmd_rmsd_covariance(gpu_ctx.handle, fr.ctypes.data, 8, 1500, 3, None, 1500, r.handle,
                                                  cov.ctypes.data, x2.ctypes.data, y2.ctypes.data, None))
    r.close()
    for f in range(8):
        x = fr[f].astype(np.float64) - fr[f].astype(np.float64).mean(0)
        y = ref.astype(np.float64) - ref.astype(np.float64).mean(0)
        np.testing.assert_allclose(cov[f].reshape(3, 3), x.T @ y, rtol=1e-6, atol=1e-2)
        np.testing.assert_allclose(x2[f], (x ** 2).sum(), rtol=1e-6)
        np.testing.assert_allclose(y2[f], (y ** 2).sum(), rtol=1e-6)


def test_plan_api_frame0_topology_subset():
    rng = np.random.default_rng(0)
    fr, ref = synth.make_trajectory(400, 12, 0.5, seed=31)
    table = {"name": ["CA" if i % 2 == 0 else "CB" for i in range(400)], "resid": list(range(400))}
    system = warp_md.System.from_arrays(table, positions0=ref)
    traj = warp_md.Trajectory.from_numpy(fr)
    sel = system.select("name CA")
    idx = np.asarray(sel.indices)
    got = warp_md.RmsdPlan(sel, reference="frame0", align=True).run(traj, system, device="cuda:0")
    exp32, _ = oracle.rmsd_frames(fr, fr[0][idx], selection=idx)
    assert got.dtype == np.float32
    np.testing.assert_allclose(got, exp32, rtol=0, atol=TOL)
    got = warp_md.RmsdPlan(sel, reference="topology").run(traj, system)
    exp32, _ = oracle.rmsd_frames(fr, ref[idx], selection=idx)
    np.testing.assert_allclose(got, exp32, rtol=0, atol=TOL)
    sub = [5, 2, -1]
    got = warp_md.RmsdPlan(sel, reference="frame0").run(traj, system, frame_indices=sub)
    frames = fr[[5, 2, 11]]
    exp32, _ = oracle.rmsd_frames(frames, frames[0][idx], selection=idx)
    np.testing.assert_allclose(got, exp32, rtol=0, atol=TOL)
    got = warp_md.RmsdPlan(system.select("all"), reference="frame0", align=False).run(traj, system)
    exp32, _ = oracle.rmsd_frames(fr, fr[0], align=False)
    np.testing.assert_allclose(got, exp32, rtol=0, atol=TOL)


def test_reference_known_answer_through_plan_api():
    # rmsd_plan_align_zero (crates/traj-engine/src/tests/analysis_smoke_tests.rs:22-37)
    pos0 = np.array([[0, 0, 0], [1, 0, 0]], np.float32)
    system = warp_md.System.from_arrays({"name": ["CA", "CA"], "resname": ["ALA", "ALA"], "resid": [1, 1]},
                                        positions0=pos0)
    vals = warp_md.RmsdPlan(system.select("name CA"), reference="topology", align=True).run(
        warp_md.Trajectory.from_numpy(pos0[None]), system)
    assert abs(vals[0]) < 1e-6


def test_streaming_workload_sampled_parity(gpu_ctx):
    """Full-size streaming workload (100,000 atoms x 10,000 frames, 12 GB on the
    device): the GPU result on every frame, checked against the oracle on a
    seeded sample of 24 frames, plus rotation/translation invariance of a few
    frames re-posed in FP64."""
    F, n = 10000, 100000
    coords, ref = synth.make_trajectory_torch(n, F, (0.05, 3.0), seed=1, device="cuda")
    r = N.Reference(gpu_ctx, ref.data_ptr(), n, 3, keepalive=ref)
    out = torch.empty(F, dtype=torch.float64, device="cuda")
    gpu_ctx.check(gpu_ctx.lib.wmd_rmsd_frames(gpu_ctx.handle, coords.data_ptr(), F, n, 3, None, n, r.handle, 1,
                                              out.data_ptr(), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    pick = np.random.default_rng(0).choice(F, 24, replace=False)
    sample = coords[torch.from_numpy(pick).cuda()].cpu().numpy()
    ref_h = ref.cpu().numpy()
    _, exp = oracle.rmsd_frames(sample, ref_h)
    np.testing.assert_allclose(got[pick], exp, rtol=0, atol=TOL)
    assert np.all(np.isfinite(got)) and got.min() > 0.05 and got.max() < 3.0 * np.sqrt(3) + 0.1
    r.close()
    del coords
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n_atoms,n_frames", [(4001, 2403), (1002, 9602), (99999, 66)])
def test_frames_across_lanes_quad_rows(gpu_ctx, n_atoms, n_frames):
    """Packed xyz frames whose stride is not a multiple of 16 bytes, enough of
    them for the frames-across-lanes kernel: it reads quad rows of 4 frames
    (odd n_atoms; n_atoms % 4 == 2) and leaves the last n_frames mod 4 frames
    (3, 2, 2 here) to the gathered kernel.  Aligned and no-fit RMSD and a
    dense prefix against the oracle (plan.rs:1093-1248) within 1e-5 A."""
    fr, ref = synth.make_trajectory(n_atoms, n_frames, (0.05, 3.0), seed=n_atoms + n_frames)
    fr[n_frames - 1] = ref  # in the gathered tail: the residual pass
    got = gpu_rmsd(gpu_ctx, fr, ref, device_io=True)
    _, exp = oracle.rmsd_frames(fr, ref)
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
    assert got[-1] < 1e-9
    raw = gpu_rmsd(gpu_ctx, fr, ref, align=False, device_io=True)
    _, expr = oracle.rmsd_frames(fr, ref, align=False)
    np.testing.assert_allclose(raw, expr, rtol=0, atol=TOL)
    k = n_atoms - 37
    got = gpu_rmsd(gpu_ctx, fr, ref[:k], device_io=True)
    _, exp = oracle.rmsd_frames(fr, ref[:k], selection=np.arange(k))
    np.testing.assert_allclose(got, exp, rtol=0, atol=TOL)
