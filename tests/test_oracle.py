"""The CPU oracle against the reference's own numbers (no GPU).

Pins: (1) golden vectors produced by the reference's numpy Kabsch helpers
(python/warp_md/analysis/_runtime.py:611-635, see tests/golden/make_golden.py);
(2) the known answers of the reference's tests for this path; (3) SVD-Kabsch ==
QCP; (4) the analytic gradient against central differences.
"""
import numpy as np
import pytest

import oracle


def _cases(golden):
    return sorted(k[len("frames_"):] for k in golden.files if k.startswith("frames_"))


def test_golden_aligned_and_raw(golden):
    for name in _cases(golden):
        fr, ref = golden["frames_" + name], golden["ref_" + name]
        o32, o64 = oracle.rmsd_frames(fr, ref, align=True)
        np.testing.assert_allclose(o64, golden["expect_aligned_" + name], rtol=0, atol=1e-12, err_msg=name)
        np.testing.assert_array_equal(o32, o64.astype(np.float32))
        r32, r64 = oracle.rmsd_frames(fr, ref, align=False)
        np.testing.assert_allclose(r64, golden["expect_raw_" + name], rtol=0, atol=1e-11, err_msg=name)


def test_golden_pairwise(golden):
    for name in _cases(golden):
        if "expect_pair_aligned_" + name not in golden.files:
            continue
        fr = golden["frames_" + name]
        _, p64 = oracle.pairwise(fr, "rms")
        np.testing.assert_allclose(p64, golden["expect_pair_aligned_" + name], rtol=0, atol=1e-12, err_msg=name)
        _, n64 = oracle.pairwise(fr, "nofit")
        np.testing.assert_allclose(n64, golden["expect_pair_raw_" + name], rtol=0, atol=1e-11, err_msg=name)


def test_known_answers_from_reference_tests():
    # rmsd_plan_align_zero (crates/traj-engine/src/tests/analysis_smoke_tests.rs:22-37)
    pos0 = np.array([[0, 0, 0], [1, 0, 0]], np.float32)
    o32, _ = oracle.rmsd_frames(pos0[None], pos0, selection=[0, 1])
    assert abs(o32[0]) < 1e-6
    # kabsch_rmsd_aligns_translated_coordinates (geometry_math.rs:299-317)
    frame = np.array([[1, 0, 0], [2, 0, 0], [1, 1, 0]], np.float32)
    ref = np.array([[3, 5, -2], [4, 5, -2], [3, 6, -2]], np.float32)
    o32, _ = oracle.rmsd_frames(frame[None], ref)
    assert o32[0] <= 1e-6
    # pairwise_rmsd_plan_basic, nofit -> sqrt(0.5) (geometry_matrix_tests.rs:1437-1459)
    fr = np.array([[[0, 0, 0], [1, 0, 0]], [[0, 0, 0], [2, 0, 0]]], np.float32)
    m32, _ = oracle.pairwise(fr, "nofit")
    assert abs(m32[0, 1] - np.sqrt(0.5)) < 1e-6 and abs(m32[1, 0] - np.sqrt(0.5)) < 1e-6
    # srmsd alias -> aligned RMSD 0.5 (python/warp_md/tests/test_pairwise_srmsd.py:40-53)
    m32, _ = oracle.pairwise(fr, "rms")
    np.testing.assert_allclose(m32[0, 1], 0.5, rtol=1e-6)
    # nofit with frame_indices [0, 2] -> sqrt(2) (test_pairwise_rmsd.py:78-103)
    fr3 = np.array([[[0, 0, 0], [1, 0, 0]], [[0, 0, 0], [2, 0, 0]], [[0, 0, 0], [3, 0, 0]]], np.float32)
    m32, _ = oracle.pairwise(fr3[[0, 2]], "nofit")
    np.testing.assert_allclose(m32[0, 1], np.sqrt(2.0), atol=1e-6)
    # symmrmsd fit=False -> [0, 0.70710677] (test_symmrmsd.py:40-53): raw RMSD vs frame 0
    r32, _ = oracle.rmsd_frames(fr, fr[0], align=False)
    np.testing.assert_allclose(r32, [0.0, 0.70710677], atol=1e-7)
    # rotation_matrix 90 degrees about z -> rmsd 0 (test_rotation_matrix.py:40-60)
    rot = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], np.float64)
    pts = np.array([[1, 0, 0], [0, 2, 0], [0, 0, 3], [1, 1, 1]], np.float32)
    o32, _ = oracle.rmsd_frames((pts @ rot.T).astype(np.float32)[None], pts)
    assert o32[0] < 1e-6


def test_empty_and_degenerate_selections():
    fr = np.random.default_rng(0).normal(size=(3, 5, 3)).astype(np.float32)
    o32, _ = oracle.rmsd_frames(fr, np.zeros((0, 3), np.float32), selection=[])
    assert np.all(o32 == 0)  # plan.rs:1166-1168
    m32, _ = oracle.pairwise(fr[:, :1], "rms")  # n_sel < 2 -> zeros (plan.rs:604-610)
    assert np.all(m32 == 0)


def test_rotation_convention_and_reflection():
    rng = np.random.default_rng(3)
    for _ in range(20):
        h = rng.normal(size=(3, 3))
        r, ss = oracle.kabsch_rotation(h)
        np.testing.assert_allclose(r @ r.T, np.eye(3), atol=1e-12)
        assert np.linalg.det(r) > 0
        # R maximises tr(R H) over rotations; value = s1 + s2 + sign(det H) s3
        s = np.linalg.svd(h, compute_uv=False)
        expect = s[0] + s[1] + (s[2] if np.linalg.det(h) > 0 else -s[2])
        assert abs(np.trace(r @ h) - expect) < 1e-10
        assert abs(ss - expect) < 1e-10


def test_qcp_matches_svd_route(golden):
    for name in _cases(golden):
        if name.startswith("collinear"):
            continue  # double root: plain QCP Newton loses digits there (the device code falls back to an SVD)
        fr, ref = golden["frames_" + name], golden["ref_" + name]
        _, o64 = oracle.rmsd_frames(fr, ref)
        for f, v in zip(fr, o64):
            assert abs(oracle.qcp_rmsd(f, ref) - v) < 1e-9
            assert abs(oracle.qcp_rmsd(f, ref, high_precision=True) - v) < 1e-9


def test_gradient_central_differences():
    from warp_md import synth

    fr, ref = synth.make_trajectory(40, 3, 0.3, 11)
    rm, g = oracle.rmsd_grad(fr, ref)
    h = 1e-4
    x64 = fr.astype(np.float64)
    rng = np.random.default_rng(1)
    for f in range(fr.shape[0]):
        for atom in rng.choice(40, 6, replace=False):
            for c in range(3):
                # central difference on an FP64 restatement of the same RMSD
                def val(delta):
                    x = x64[f].copy()
                    x[atom, c] += delta
                    xc = x - x.mean(0)
                    yc = ref.astype(np.float64) - ref.astype(np.float64).mean(0)
                    u, s, vt = np.linalg.svd(xc.T @ yc)
                    d = np.sign(np.linalg.det(vt.T @ u.T))
                    msd = ((xc ** 2).sum() + (yc ** 2).sum() - 2 * (s[0] + s[1] + d * s[2])) / len(x)
                    return np.sqrt(max(msd, 0))
                fd = (val(h) - val(-h)) / (2 * h)
                assert abs(fd - g[f, atom, c]) < 1e-6 * max(1.0, abs(fd)), (f, atom, c, fd, g[f, atom, c])
