"""The oracle's superposition (AlignPlan / SuperposePlan semantics) on the CPU.

Pins: (1) the known answers of the reference's tests for these plans
(python/warp_md/tests/test_superpose.py, test_align.py, test_rotation_matrix.py:
a 90-degree rotation plus a translation is undone exactly; the rotation of
frame 1 is rot^T); (2) the golden vectors of the reference's numpy Kabsch
(python/warp_md/analysis/_runtime.py:611-628, tests/golden/make_golden.py):
applying the oracle's FP64 transform to the selection reproduces the
reference's minimum RMSD; (3) the weighted form against an independent numpy
restatement of kabsch_rotation_weighted (geometry_math.rs:235-300).
"""
import numpy as np

import oracle

ROT90 = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
TRI = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])


def _apply64(xf, coords):
    r = xf[:, :9].reshape(-1, 3, 3)
    return np.einsum("fij,faj->fai", r, coords.astype(np.float64)) + xf[:, None, 9:12]


def test_known_answers_from_reference_tests():
    # test_superpose_all_frames / test_align_basic: frame1 = ref @ rot^T + (2, 3, 0)
    frame1 = TRI @ ROT90.T + np.array([2.0, 3.0, 0.0])
    coords = np.stack([TRI, frame1]).astype(np.float32)
    xf, out = oracle.superpose(coords, coords[0])
    np.testing.assert_allclose(out[0], TRI, atol=1e-5)
    np.testing.assert_allclose(out[1], TRI, atol=1e-5)
    # test_rotation_matrix_basic: frame1 = ref @ rot^T -> mats[1] = rot^T, mats[0] = I
    coords = np.stack([TRI, TRI @ ROT90.T]).astype(np.float32)
    xf, _ = oracle.superpose(coords, coords[0], apply=False)
    np.testing.assert_allclose(xf[0, :9].reshape(3, 3), np.eye(3), atol=1e-6)
    np.testing.assert_allclose(xf[1, :9].reshape(3, 3), ROT90.T, atol=1e-6)


def test_golden_transform_reaches_reference_minimum(golden):
    names = sorted(k[len("frames_"):] for k in golden.files if k.startswith("frames_"))
    for name in names:
        fr, ref = golden["frames_" + name], golden["ref_" + name]
        xf, out = oracle.superpose(fr, ref)
        moved = _apply64(xf, fr)
        rmsd = np.sqrt(((moved - ref.astype(np.float64)) ** 2).sum(axis=(1, 2)) / fr.shape[1])
        np.testing.assert_allclose(rmsd, golden["expect_aligned_" + name], rtol=0, atol=1e-9, err_msg=name)
        # the float32 output is the FP64 transform rounded once
        assert np.abs(out - moved).max() <= np.abs(moved).max() * 2.0 ** -23


def _numpy_weighted_kabsch(x, y, w):
    cx = (x * w[:, None]).sum(0) / w.sum()
    cy = (y * w[:, None]).sum(0) / w.sum()
    h = ((x - cx) * w[:, None]).T @ (y - cy)
    u, _s, vt = np.linalg.svd(h)
    r = vt.T @ u.T
    if np.linalg.det(r) < 0:
        vt[-1] *= -1
        r = vt.T @ u.T
    return r, cy - r @ cx


def test_weighted_against_numpy_restatement():
    rng = np.random.default_rng(4)
    from warp_md import synth

    fr, ref = synth.make_trajectory(120, 6, 0.8, 11)
    w = rng.uniform(1.0, 16.0, 120).astype(np.float32)
    sel = np.sort(rng.choice(120, 50, replace=False)).astype(np.uint32)
    xf, out = oracle.superpose(fr, ref[sel], selection=sel, weights=w[sel])
    for f in range(fr.shape[0]):
        r, t = _numpy_weighted_kabsch(fr[f][sel].astype(np.float64), ref[sel].astype(np.float64),
                                      w[sel].astype(np.float64))
        np.testing.assert_allclose(xf[f, :9].reshape(3, 3), r, atol=1e-10)
        np.testing.assert_allclose(xf[f, 9:], t, atol=1e-8)
    # equal weights give the unweighted transform
    xf1, _ = oracle.superpose(fr, ref, weights=np.full(120, 2.5, np.float32), apply=False)
    xf0, _ = oracle.superpose(fr, ref, apply=False)
    np.testing.assert_allclose(xf1, xf0, atol=1e-9)


def test_norotate_and_empty_selection():
    from warp_md import synth

    fr, ref = synth.make_trajectory(40, 3, 0.5, 2)
    xf, out = oracle.superpose(fr, ref, norotate=True)
    np.testing.assert_array_equal(xf[:, :9], np.tile(np.eye(3).reshape(1, 9), (3, 1)))
    np.testing.assert_allclose(xf[:, 9:], ref.astype(np.float64).mean(0) - fr.astype(np.float64).mean(1), atol=1e-9)
    xf, out = oracle.superpose(fr, np.zeros((0, 3), np.float32), selection=np.zeros(0, np.uint32))
    np.testing.assert_array_equal(xf[:, :9], np.tile(np.eye(3).reshape(1, 9), (3, 1)))
    np.testing.assert_array_equal(xf[:, 9:], 0.0)
    np.testing.assert_array_equal(out, fr)
