"""All-pairs RMSD matrix on the GPU against the oracle's restatement of
PairwiseRmsdPlan::finalize (plan.rs:593-674).

Tolerances (max abs error vs the FP64 oracle; outputs are float32 like the
reference's, so a relative 1e-7 for the float32 rounding of large values is
added to each):
  fp64 : 1e-5 A   (FP64 covariance tiles, exact up to the float32 output)
  i8x3 : 1e-4 A   (24-bit fixed point, the eight limb products other than lo x lo in exact
                   int32 accumulation; pairs below 0.01 A recomputed exactly in FP64)
  i8x2 : 5e-4 A   (16-bit fixed point)
  fp32 : 2e-2 A   (plain FP32 accumulation; measured error is reported by bench.py)
"""
import numpy as np
import pytest

import oracle
import warp_md
from warp_md import _native as N
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-5, "i8x3": 1e-4, "i8x2": 5e-4, "fp32": 2e-2}
MODES = ["fp64", "fp32", "i8x3", "i8x2"]


def gpu_pairwise(ctx, frames, metric="rms", mode="fp64", sel=None, device_io=False):
    from warp_md.plans import _PAIR_MODES

    fr = np.ascontiguousarray(frames, np.float32)
    F, n_atoms = fr.shape[0], fr.shape[1]
    n_sel = n_atoms if sel is None else len(sel)
    m = N.PAIR_RMS if metric == "rms" else N.PAIR_NOFIT
    if device_io:
        d = torch.from_numpy(fr).cuda()
        out = torch.empty(F, F, dtype=torch.float32, device="cuda")
        ds = None if sel is None else torch.from_numpy(np.asarray(sel, np.int32)).cuda()
        ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, d.data_ptr(), F, n_atoms, 3,
                                            None if ds is None else ds.data_ptr(), n_sel, m, _PAIR_MODES[mode],
                                            out.data_ptr(), None))
        torch.cuda.synchronize()
        return out.cpu().numpy()
    out = np.empty((F, F), np.float32)
    s = None if sel is None else np.ascontiguousarray(sel, np.uint32)
    ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, fr.ctypes.data, F, n_atoms, 3, N.ptr(s), n_sel, m,
                                        _PAIR_MODES[mode], out.ctypes.data, None))
    return out


def _supported(ctx, mode):
    fr = np.zeros((2, 3, 3), np.float32)
    out = np.empty((2, 2), np.float32)
    from warp_md.plans import _PAIR_MODES

    rc = ctx.lib.wmd_pairwise_rmsd(ctx.handle, fr.ctypes.data, 2, 3, 3, None, 3, 0, _PAIR_MODES[mode],
                                   out.ctypes.data, None)
    return rc != N.WMD_ERR_UNSUPPORTED


@pytest.mark.parametrize("mode", MODES)
def test_golden_pairwise(gpu_ctx, golden, mode):
    if not _supported(gpu_ctx, mode):
        pytest.skip(f"{mode} not built")
    for name in sorted(k[7:] for k in golden.files if k.startswith("frames_")):
        if "expect_pair_aligned_" + name not in golden.files:
            continue
        fr = golden["frames_" + name]
        got = gpu_pairwise(gpu_ctx, fr, "rms", mode)
        np.testing.assert_allclose(got, golden["expect_pair_aligned_" + name], rtol=1e-7, atol=TOL[mode], err_msg=name)
        got = gpu_pairwise(gpu_ctx, fr, "nofit", mode)
        np.testing.assert_allclose(got, golden["expect_pair_raw_" + name], rtol=1e-7, atol=TOL[mode], err_msg=name)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("F,n", [(2, 2), (3, 5), (33, 17), (129, 100), (300, 257)])
def test_drift_shapes(gpu_ctx, mode, F, n):
    if not _supported(gpu_ctx, mode):
        pytest.skip(f"{mode} not built")
    fr = synth.make_drift_trajectory(n, F, 0.1, seed=F + n)
    got = gpu_pairwise(gpu_ctx, fr, "rms", mode, device_io=True)
    _, exp = oracle.pairwise(fr, "rms")
    assert np.all(np.diag(got) == 0)
    np.testing.assert_array_equal(got, got.T)
    np.testing.assert_allclose(got, exp, rtol=1e-7, atol=TOL[mode])


@pytest.mark.parametrize("mode", MODES)
def test_allpairs_subblock(gpu_ctx, mode):
    """All-pairs workload recipe (slow drift + random rigid motions), 1,000
    atoms; errors on a 512 x 512 block against the FP64 oracle."""
    if not _supported(gpu_ctx, mode):
        pytest.skip(f"{mode} not built")
    fr = synth.make_drift_trajectory(1000, 640, 0.1, seed=3)
    got = gpu_pairwise(gpu_ctx, fr, "rms", mode, device_io=True)
    _, exp = oracle.pairwise(fr, "rms", block=(0, 512, 128, 640))
    err = np.abs(got[0:512, 128:640] - exp)
    assert err.max() <= TOL[mode], (mode, err.max(), np.sqrt((err ** 2).mean()))


def test_selection_and_small_selections(gpu_ctx):
    fr = synth.make_drift_trajectory(300, 40, 0.1, seed=8)
    sel = np.arange(1, 300, 2)
    got = gpu_pairwise(gpu_ctx, fr, "rms", "fp64", sel=sel)
    _, exp = oracle.pairwise(fr[:, sel], "rms")
    np.testing.assert_allclose(got, exp, rtol=1e-7, atol=1e-5)
    one = gpu_pairwise(gpu_ctx, fr, "rms", "fp64", sel=[7])
    assert np.all(one == 0)  # n_sel < 2 -> zeros (plan.rs:604-610)


def test_plan_api_known_answers():
    coords = np.array([[[0, 0, 0], [1, 0, 0]], [[0, 0, 0], [2, 0, 0]], [[0, 0, 0], [3, 0, 0]]], np.float32)
    system = warp_md.System.from_arrays({"name": ["DA", "AC"], "resid": [1, 2]}, positions0=coords[0])
    traj = warp_md.Trajectory.from_numpy(coords)
    sel = system.select("resid 1:2")
    m = warp_md.PairwiseRmsdPlan(sel, metric="nofit").run(traj, system, frame_indices=[0, 1])
    assert abs(m[0, 1] - np.sqrt(0.5)) < 1e-6 and abs(m[1, 0] - np.sqrt(0.5)) < 1e-6
    m = warp_md.PairwiseRmsdPlan(sel, metric="nofit").run(traj, system, frame_indices=[0, 2])
    np.testing.assert_allclose(m[0, 1], np.sqrt(2.0), atol=1e-6)
    from warp_md.analysis.rmsd import pairwise_rmsd

    m = pairwise_rmsd(warp_md.Trajectory.from_numpy(coords[:2]), system, mask="all", metric="srmsd")
    np.testing.assert_allclose(m[0, 1], 0.5, rtol=1e-6)
    half = pairwise_rmsd(traj, system, mask="all", metric="nofit", mat_type="half")
    assert half.shape == (3,)


# ---------------------------------------------------------------------------
# metric "dme" (distance-matrix error): the kernel sums in the reference's
# order with the reference's roundings, so it is compared bit for bit with the
# oracle (tolerance 0), and cross-checked for host/device inputs.
# ---------------------------------------------------------------------------

def gpu_dme(ctx, frames, sel=None, box=None, device_io=False, stride=3):
    fr = np.ascontiguousarray(frames, np.float32)
    if stride == 4:
        fr = np.ascontiguousarray(np.concatenate([fr, np.full(fr.shape[:2] + (1,), 7.0, np.float32)], axis=2))
    F, n_atoms = fr.shape[0], fr.shape[1]
    n_sel = n_atoms if sel is None else len(sel)
    b = None if box is None else np.array(np.broadcast_to(np.asarray(box, np.float32), (F, 3)), order="C")
    if device_io:
        d = torch.from_numpy(fr).cuda()
        out = torch.empty(F, F, dtype=torch.float32, device="cuda")
        ds = None if sel is None else torch.from_numpy(np.asarray(sel, np.int32)).cuda()
        db = None if b is None else torch.from_numpy(b).cuda()
        ctx.check(ctx.lib.wmd_pairwise_dme(ctx.handle, d.data_ptr(), F, n_atoms, stride,
                                           None if ds is None else ds.data_ptr(), n_sel,
                                           None if db is None else db.data_ptr(), out.data_ptr(), None))
        torch.cuda.synchronize()
        return out.cpu().numpy()
    out = np.empty((F, F), np.float32)
    s = None if sel is None else np.ascontiguousarray(sel, np.uint32)
    ctx.check(ctx.lib.wmd_pairwise_dme(ctx.handle, fr.ctypes.data, F, n_atoms, stride, N.ptr(s), n_sel, N.ptr(b),
                                       out.ctypes.data, None))
    return out


@pytest.mark.parametrize("F,n", [(1, 5), (31, 7), (32, 40), (33, 2), (65, 33), (100, 64)])
def test_dme_matches_oracle(gpu_ctx, F, n):
    fr = synth.make_drift_trajectory(n, F, 0.3, seed=F + n)
    got = gpu_dme(gpu_ctx, fr)
    want, _ = oracle.pairwise_dme(fr)
    np.testing.assert_array_equal(got, want)
    assert (np.diag(got) == 0).all()


@pytest.mark.parametrize("device_io", [False, True])
def test_dme_selection_pbc_and_stride(gpu_ctx, device_io):
    rng = np.random.default_rng(3)
    fr = rng.uniform(0, 12, size=(45, 60, 3)).astype(np.float32)  # atoms spread over the box
    sel = rng.permutation(60)[:37]  # unsorted selection
    box = np.stack([np.full(45, 12.0), np.full(45, 11.5), np.linspace(10.0, 13.0, 45)], 1).astype(np.float32)
    for b in (None, box, np.array([12.0, 0.0, 12.0], np.float32)):
        want, _ = oracle.pairwise_dme(fr[:, sel], box=b)
        got = gpu_dme(gpu_ctx, fr, sel=sel, box=b, device_io=device_io)
        np.testing.assert_array_equal(got, want)
        got4 = gpu_dme(gpu_ctx, fr, sel=sel, box=b, device_io=device_io, stride=4)
        np.testing.assert_array_equal(got4, want)


def test_dme_small_selection_and_metric_code(gpu_ctx):
    fr = synth.make_drift_trajectory(20, 9, 0.3, seed=5)
    out = np.full((9, 9), np.nan, np.float32)
    gpu_ctx.check(gpu_ctx.lib.wmd_pairwise_dme(gpu_ctx.handle, fr.ctypes.data, 9, 20, 3,
                                               N.ptr(np.array([4], np.uint32)), 1, None, out.ctypes.data, None))
    assert (out == 0).all()  # n_sel < 2 -> zeros (plan.rs:604-610)
    # wmd_pairwise_rmsd with metric WMD_PAIR_DME is the same call without a box
    from warp_md.plans import _PAIR_MODES

    out2 = np.empty((9, 9), np.float32)
    gpu_ctx.check(gpu_ctx.lib.wmd_pairwise_rmsd(gpu_ctx.handle, fr.ctypes.data, 9, 20, 3, None, 20, N.PAIR_DME,
                                                _PAIR_MODES["fp64"], out2.ctypes.data, None))
    np.testing.assert_array_equal(out2, oracle.pairwise_dme(fr)[0])


def test_dme_plan_api():
    coords = np.array([[[0, 0, 0], [1, 0, 0]], [[0, 0, 0], [1, 0, 0]]], np.float32)
    system = warp_md.System.from_arrays({"name": ["A", "B"], "resid": [1, 2]}, positions0=coords[0])
    from warp_md.analysis.rmsd import pairwise_rmsd

    # the reference's test_pairwise_rmsd_dme_zero_for_identical (test_pairwise_rmsd.py:64-75)
    mat = pairwise_rmsd(warp_md.Trajectory.from_numpy(coords), system, mask="all", metric="dme", mat_type="full")
    assert np.allclose(mat[0, 1], 0.0)
    fr = synth.make_drift_trajectory(30, 12, 0.5, seed=9)
    sys30 = warp_md.System.from_arrays({"name": ["CA"] * 30, "resid": list(range(1, 31))}, positions0=fr[0])
    sel = sys30.select("resid 3:27")
    idx = np.asarray(sel.indices)
    box = np.array([40.0, 35.0, 50.0], np.float32)
    traj = warp_md.Trajectory.from_numpy(fr, box=box)
    m = warp_md.PairwiseRmsdPlan(sel, metric="dme", pbc="orthorhombic").run(traj, sys30, frame_indices=[0, 5, 11])
    want, _ = oracle.pairwise_dme(fr[[0, 5, 11]][:, idx], box=box)
    np.testing.assert_array_equal(m, want)
    m = warp_md.PairwiseRmsdPlan(sel, metric="dme").run(traj, sys30)
    np.testing.assert_array_equal(m, oracle.pairwise_dme(fr[:, idx])[0])
    # length_scale multiplies the matrix (python/warp_md/analysis/rmsd.py:197)
    half = pairwise_rmsd(traj, sys30, mask="resid 3:27", metric="dme", mat_type="half", length_scale=0.1)
    full = oracle.pairwise_dme(fr[:, idx])[0] * np.float32(0.1)
    np.testing.assert_array_equal(half, full[np.triu_indices(12, k=1)])


def test_i8x3_full_all_pairs_workload_blocks_against_oracle():
    """The all-pairs workload at full size: 20,000 frames x 1,000 atoms of
    slow random drift (N(0, 0.1 A) per atom per frame) under random rigid
    motions, through the tensor-core i8x3 form, device-resident.  Checked
    against the FP64 oracle (plan.rs:593-674) on the leading 512 x 512 block
    and on a 512-frame block strided over the whole trajectory (every 39th
    frame, pairs up to ~20,000 frames apart), at the 1e-4 A bar."""
    ctx = N.context(0)
    if not _supported(ctx, "i8x3"):
        pytest.skip("tensor-core form not supported on this device")
    from warp_md.plans import _PAIR_MODES

    F, n = 20000, 1000
    d = synth.make_drift_trajectory_torch(n, F, 0.1, seed=3, device="cuda")
    out = torch.empty(F, F, dtype=torch.float32, device="cuda")
    ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, d.data_ptr(), F, n, 3, None, n, N.PAIR_RMS,
                                        _PAIR_MODES["i8x3"], out.data_ptr(), None))
    torch.cuda.synchronize()
    assert bool(torch.isfinite(out).all().item())
    assert float(out.diagonal().abs().max().item()) == 0.0
    for idx in (np.arange(512), np.arange(0, F, 39)[:512]):
        ti = torch.from_numpy(idx).cuda()
        got = out.index_select(0, ti).index_select(1, ti).cpu().numpy()
        _, exact = oracle.pairwise(d.index_select(0, ti).cpu().numpy(), "rms")
        err = np.abs(got - exact)
        assert err.max() <= TOL["i8x3"] + 1e-7 * np.abs(exact).max(), (idx[:3], float(err.max()))
    # symmetric fill, as the reference mirrors the upper triangle
    blk = out[:2000, :2000]
    assert bool(torch.equal(blk, blk.t()))
    del out, d
    torch.cuda.empty_cache()


@pytest.mark.parametrize("mode", MODES)
def test_parts_are_disjoint_and_sum_to_the_full_matrix(mode):
    """wmd_pairwise_rmsd_part: the tile-row partition of the i < j loop
    (plan.rs:593-674) that the multi-GPU assembly sums.  For 2, 3 and 7 parts,
    no entry is written by two parts and the sum of the parts is the
    single-call matrix bit for bit."""
    from warp_md.plans import _PAIR_MODES

    ctx = N.context(0)
    if not _supported(ctx, mode):
        pytest.skip(f"{mode} not supported on this device")
    d = synth.make_drift_trajectory(120, 300, 0.1, seed=31)
    x = torch.from_numpy(d).cuda()
    F = d.shape[0]
    full = torch.empty(F, F, dtype=torch.float32, device="cuda")
    ctx.check(ctx.lib.wmd_pairwise_rmsd(ctx.handle, x.data_ptr(), F, 120, 3, None, 120, N.PAIR_RMS,
                                        _PAIR_MODES[mode], full.data_ptr(), None))
    for parts in (2, 3, 7):
        total = torch.zeros_like(full)
        written = torch.zeros(F, F, dtype=torch.int32, device="cuda")
        for part in range(parts):
            out = torch.full((F, F), -1.0, dtype=torch.float32, device="cuda")
            ctx.check(ctx.lib.wmd_pairwise_rmsd_part(ctx.handle, x.data_ptr(), F, 120, 3, None, 120, N.PAIR_RMS,
                                                     _PAIR_MODES[mode], part, parts, out.data_ptr(), None))
            total += out
            written += (out != 0).int()
        torch.cuda.synchronize()
        assert int(written.max().item()) == 1
        assert bool(torch.equal(total, full)), (mode, parts)
    bad = ctx.lib.wmd_pairwise_rmsd_part(ctx.handle, x.data_ptr(), F, 120, 3, None, 120, N.PAIR_RMS,
                                         _PAIR_MODES[mode], 3, 3, full.data_ptr(), None)
    assert bad == N.WMD_ERR_INVALID_ARG


def _near_identical(F, n, step, seed):
    """Frames that differ by ~step A per coordinate from frame 0, each under a
    random rigid motion: every pair is below the 0.01 A refine threshold."""
    rng = np.random.default_rng(seed)
    base = synth.make_trajectory(n, 1, 0.0, seed)[1]
    out = np.empty((F, n, 3), np.float32)
    for f in range(F):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        noisy = base + rng.normal(0, step, base.shape)
        out[f] = (noisy @ R.T + rng.normal(0, 10, 3)).astype(np.float32)
    return out


@pytest.mark.parametrize("metric", ["rms", "nofit"])
def test_i8x3_pairs_below_refine_threshold_are_exact(metric):
    """3 limbs leave the lo x lo limb product out of the tensor-core sums; the
    pairs whose RMSD then comes out below 0.01 A are recomputed in FP64 from
    the coordinates.  Frames within ~1e-3 A of each other (a duplicate
    included): every off-diagonal pair is refined and agrees with the oracle
    to 2e-6 A (FP64 against FP64, float32 output), the duplicate pair to 0."""
    ctx = N.context(0)
    if not _supported(ctx, "i8x3"):
        pytest.skip("tensor-core form not supported on this device")
    fr = _near_identical(96, 700, 6e-4, seed=5)
    fr[17] = fr[3]
    if metric == "nofit":  # no superposition: identical placement, small displacements
        fr = np.repeat(fr[:1], 96, axis=0) + np.random.default_rng(6).normal(0, 6e-4, fr.shape).astype(np.float32)
        fr[17] = fr[3]
    got = gpu_pairwise(ctx, fr, metric, "i8x3", device_io=True)
    _, exp = oracle.pairwise(fr, metric)
    off = ~np.eye(96, dtype=bool)
    assert exp[off].max() < 0.01
    np.testing.assert_allclose(got, exp, rtol=1e-6, atol=2e-6)
    assert got[3, 17] < 2e-6 and got[17, 3] < 2e-6


def test_i8x3_refine_list_overflow_scans_the_matrix():
    """More flagged pairs than the list holds (1,600 near-identical frames:
    1,279,200 pairs against a list of 2^20): the refine pass then finds them
    in the matrix itself; the result equals the oracle on a 300-frame block."""
    ctx = N.context(0)
    if not _supported(ctx, "i8x3"):
        pytest.skip("tensor-core form not supported on this device")
    F = 1600
    fr = _near_identical(F, 200, 5e-4, seed=9)
    got = gpu_pairwise(ctx, fr, "rms", "i8x3", device_io=True)
    idx = np.r_[np.arange(150), np.arange(F - 150, F)]
    _, exp = oracle.pairwise(fr[idx], "rms")
    np.testing.assert_allclose(got[np.ix_(idx, idx)], exp, rtol=1e-6, atol=2e-6)
