"""Superposition on the GPU (wmd_superpose_transforms / wmd_superpose and the
AlignPlan, RotationMatrixPlan, SuperposePlan, SuperposeTrajectoryPlan and
analysis wrappers) against the oracle.

Tolerances: the transform's rotation within 1e-6 of the oracle's FP64 value
(the result is float32), its translation within 2 float32 ulps; moved
coordinates within one float32 ulp of the oracle's FP64 transform applied to
the same input (both round R x + t once), plus 1e-9 A for values near zero.
"""
import numpy as np
import pytest

import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _check_xf(got, want):
    np.testing.assert_allclose(got[:, :9], want[:, :9], rtol=0, atol=1e-6)
    t = want[:, 9:]
    assert np.all(np.abs(got[:, 9:] - t) <= 2 * np.spacing(np.abs(t).astype(np.float32)) + 1e-6)


def _check_coords(got, want):
    tol = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64) * 1.01 + 1e-9
    bad = np.abs(got.astype(np.float64) - want.astype(np.float64)) > tol
    assert not bad.any(), (np.abs(got - want).max(), int(bad.sum()))


def _ctx():
    from warp_md import _native as N

    return N, N.context(0)


def _superpose(coords, ref, sel=None, weights=None, norotate=False, device_io=False, stride=3):
    N, ctx = _ctx()
    F, n_atoms = coords.shape[0], coords.shape[1]
    r = N.Reference.from_numpy(ctx, ref, weights=weights)
    sel_arr = None if sel is None else np.ascontiguousarray(sel, np.uint32)
    n_sel = ref.shape[0]
    try:
        if device_io:
            x = torch.from_numpy(np.ascontiguousarray(coords)).cuda()
            out = torch.empty(F, n_atoms, 3, device="cuda")
            xf = torch.empty(F, 12, device="cuda")
            s = torch.from_numpy(sel_arr.astype(np.int32)).cuda() if sel_arr is not None else None
            ctx.check(ctx.lib.wmd_superpose(ctx.handle, x.data_ptr(), F, n_atoms, stride,
                                            None if s is None else s.data_ptr(), n_sel, r.handle, int(norotate),
                                            out.data_ptr(), xf.data_ptr(), torch.cuda.current_stream().cuda_stream))
            torch.cuda.synchronize()
            return xf.cpu().numpy(), out.cpu().numpy()
        out = np.empty((F, n_atoms, 3), np.float32)
        xf = np.empty((F, 12), np.float32)
        c = np.ascontiguousarray(coords, np.float32)
        ctx.check(ctx.lib.wmd_superpose(ctx.handle, c.ctypes.data, F, n_atoms, stride, N.ptr(sel_arr), n_sel,
                                        r.handle, int(norotate), out.ctypes.data, xf.ctypes.data, None))
        return xf, out
    finally:
        r.close()


def _oracle_moved(xf64, coords):
    r = xf64[:, :9].reshape(-1, 3, 3)
    c = coords[..., :3].astype(np.float64)
    return (np.einsum("fij,faj->fai", r, c) + xf64[:, None, 9:12]).astype(np.float32)


@pytest.mark.parametrize("device_io", [False, True])
def test_superpose_dense_matches_oracle(device_io):
    fr, ref = synth.make_trajectory(3000, 12, 0.5, 21)
    xf, out = _superpose(fr, ref, device_io=device_io)
    oxf, _ = oracle.superpose(fr, ref)
    _check_xf(xf, oxf)
    _check_coords(out, _oracle_moved(oxf, fr))


def test_superpose_selection_weights_and_ragged_sizes():
    rng = np.random.default_rng(3)
    # (1025, 300) and (8000, 4000), at least 1/4 dense, also stream their atom span with weights; the
    # full selection of 4096 atoms streams the weighted dense selection
    for n_atoms, F, n_sel in [(7, 3, 4), (1025, 5, 300), (5000, 4, 1100), (40000, 2, 9000), (8000, 37, 4000),
                              (4096, 33, 4096)]:
        fr, ref_all = synth.make_trajectory(n_atoms, F, 0.7, n_atoms)
        sel = np.sort(rng.choice(n_atoms, n_sel, replace=False)).astype(np.uint32)
        w = rng.uniform(1.0, 32.0, n_atoms).astype(np.float32)
        for weights in (None, w[sel]):
            xf, out = _superpose(fr, ref_all[sel], sel=sel, weights=weights)
            oxf, _ = oracle.superpose(fr, ref_all[sel], selection=sel, weights=weights)
            _check_xf(xf, oxf)
            _check_coords(out, _oracle_moved(oxf, fr))


def test_superpose_stride4_and_norotate():
    fr, ref = synth.make_trajectory(777, 6, 0.4, 5)
    fr4 = np.concatenate([fr, np.zeros(fr.shape[:2] + (1,), np.float32)], axis=2)
    xf, out = _superpose(fr4, ref, stride=4)
    oxf, _ = oracle.superpose(fr4, ref)
    _check_xf(xf, oxf)
    _check_coords(out, _oracle_moved(oxf, fr4))
    xf, out = _superpose(fr, ref, norotate=True)
    oxf, _ = oracle.superpose(fr, ref, norotate=True)
    np.testing.assert_array_equal(xf[:, :9], np.tile(np.eye(3, dtype=np.float32).reshape(1, 9), (6, 1)))
    _check_xf(xf, oxf)
    _check_coords(out, _oracle_moved(oxf, fr))


def test_superpose_empty_selection_and_zero_weights():
    fr, ref = synth.make_trajectory(50, 3, 0.4, 6)
    xf, out = _superpose(fr, np.zeros((0, 3), np.float32), sel=np.zeros(0, np.uint32))
    np.testing.assert_array_equal(out, fr)
    np.testing.assert_array_equal(xf[:, 9:], 0.0)
    xf, out = _superpose(fr, ref, weights=np.zeros(50, np.float32))
    np.testing.assert_array_equal(out, fr)


def test_weighted_reference_rejected_by_rmsd_entry_points():
    N, ctx = _ctx()
    fr, ref = synth.make_trajectory(30, 2, 0.4, 7)
    r = N.Reference.from_numpy(ctx, ref, weights=np.ones(30, np.float32))
    out = np.empty(2)
    rc = ctx.lib.wmd_rmsd_frames(ctx.handle, fr.ctypes.data, 2, 30, 3, None, 30, r.handle, 1, out.ctypes.data, None)
    assert rc == N.WMD_ERR_INVALID_ARG
    r.close()


def test_plans_match_oracle_and_reference_semantics():
    import warp_md

    rng = np.random.default_rng(8)
    n = 400
    fr, ref = synth.make_trajectory(n, 9, 0.6, 30)
    masses = rng.uniform(1.0, 16.0, n).astype(np.float32)
    system = warp_md.System.from_arrays({"name": ["CA" if i % 3 == 0 else "C" for i in range(n)], "mass": masses},
                                        positions0=ref)
    traj = warp_md.Trajectory.from_numpy(fr, time_ps=np.arange(9, dtype=np.float32))
    sel = system.select("name CA")
    idx = sel.as_array()
    # AlignPlan: (frames, 12)
    rows = warp_md.AlignPlan(sel, mass=True).run(traj, system)
    oxf, _ = oracle.superpose(fr, ref[idx], selection=idx, weights=masses[idx], apply=False)
    assert rows.shape == (9, 12) and rows.dtype == np.float32
    _check_xf(rows, oxf)
    # RotationMatrixPlan with a frame subset and frame0 reference
    mats = warp_md.RotationMatrixPlan(sel, reference="frame0").run(traj, system, frame_indices=[-1, 2, 5])
    sub = np.array([8, 2, 5])
    oxf, _ = oracle.superpose(fr[sub], fr[8][idx], selection=idx, apply=False)
    np.testing.assert_allclose(mats, oxf[:, :9], atol=1e-6)
    # SuperposePlan: flat series of frames x atoms x 3
    flat = warp_md.SuperposePlan(sel).run(traj, system)
    oxf, _ = oracle.superpose(fr, ref[idx], selection=idx)
    _check_coords(flat.reshape(9, n, 3), _oracle_moved(oxf, fr))
    # SuperposeTrajectoryPlan: payload dict
    payload = warp_md.SuperposeTrajectoryPlan(sel).run(traj, system, frame_indices=[0, 4])
    assert payload["coords"].shape == (2, n, 3) and payload["box"] is None
    np.testing.assert_array_equal(payload["time_ps"], np.array([0.0, 4.0], np.float32))
    _check_coords(payload["coords"], _oracle_moved(oxf[[0, 4]], fr[[0, 4]]))


class _DummySelection:
    def __init__(self, indices):
        self.indices = indices


class _DummySystem:
    def __init__(self, n_atoms):
        self._atoms = {"name": ["CA"] * n_atoms, "resname": ["ALA"] * n_atoms, "resid": [1] * n_atoms,
                       "chain_id": [0] * n_atoms, "mass": [1.0] * n_atoms}

    def atom_table(self):
        return self._atoms

    def select(self, _mask):
        return _DummySelection(range(len(self._atoms["name"])))


class _DummyTraj:
    def __init__(self, coords):
        self._coords = coords
        self._used = False

    def read_chunk(self, _max_frames=128):
        if self._used:
            return None
        self._used = True
        return {"coords": self._coords}


ROT90 = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
TRI = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])


def test_analysis_wrappers_reference_known_answers():
    """The reference's own test cases (test_superpose.py, test_align.py,
    test_rotation_matrix.py) through this build's wrappers."""
    from warp_md.analysis.align import align, superpose
    from warp_md.analysis.rotation import rotation_matrix

    trans = np.array([2.0, 3.0, 0.0])
    frame1 = TRI @ ROT90.T + trans
    coords = np.stack([TRI, frame1], axis=0)
    out = superpose(_DummyTraj(coords), _DummySystem(3), mask="protein", ref=0).read_chunk()["coords"]
    assert np.allclose(out[0], TRI, atol=1e-5) and np.allclose(out[1], TRI, atol=1e-5)
    out = align(_DummyTraj(coords), _DummySystem(3), mask="protein", ref=0).read_chunk()["coords"]
    assert np.allclose(out[0], TRI, atol=1e-5) and np.allclose(out[1], TRI, atol=1e-5)
    frame2 = TRI + np.array([5.0, 0.0, 0.0])
    coords3 = np.stack([TRI, frame1, frame2], axis=0)
    out = superpose(_DummyTraj(coords3), _DummySystem(3), mask="protein", ref=0,
                    frame_indices=[1]).read_chunk()["coords"]
    assert np.allclose(out[1], TRI, atol=1e-5) and np.allclose(out[2], frame2, atol=1e-5)
    coords = np.stack([TRI, TRI @ ROT90.T], axis=0).astype(np.float32)
    mats, rmsd = rotation_matrix(_DummyTraj(coords), _DummySystem(3), mask="all", ref=0, with_rmsd=True)
    assert mats.shape == (2, 3, 3)
    np.testing.assert_allclose(mats[0], np.eye(3), rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(mats[1], ROT90.T, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(rmsd[0], 0.0, rtol=1e-6, atol=1e-6)


def test_superpose_large_frames_host_chunks():
    """Frames larger than one host chunk buffer and a multi-chunk trajectory:
    100,000 atoms x 300 frames (360 MB in and out) through host pointers."""
    fr, ref = synth.make_trajectory_torch(100_000, 300, (0.05, 3.0), seed=12, device="cuda")
    host = fr.cpu().numpy()
    xf, out = _superpose(host, ref.cpu().numpy())
    sample = np.arange(0, 300, 37)
    oxf, _ = oracle.superpose(host[sample], ref.cpu().numpy())
    _check_xf(xf[sample], oxf)
    _check_coords(out[sample], _oracle_moved(oxf, host[sample]))


def test_superpose_weighted_quad_rows_odd_atoms():
    """Mass-weighted transforms over every atom of 2,001-atom packed frames
    (stride not a multiple of 16 bytes): the frames-across-lanes kernel on
    quad rows plus the gathered tail, against the oracle's weighted Kabsch."""
    n, F = 2001, 4801
    fr, ref = synth.make_trajectory(n, F, 0.4, 77)
    w = np.random.default_rng(7).uniform(1.0, 16.0, n).astype(np.float32)
    xf, out = _superpose(fr, ref, weights=w, device_io=True)
    pick = np.r_[0:40, F - 40:F]
    oxf, _ = oracle.superpose(fr[pick], ref, weights=w)
    _check_xf(xf[pick], oxf)
    _check_coords(out[pick], _oracle_moved(oxf, fr[pick]))
