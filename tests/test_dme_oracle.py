"""The oracle's restatement of PairwiseRmsdPlan metric "dme" (plan.rs:612-645,
pair_distances_compact plan.rs:1279-1302, apply_pbc pbc_math.rs:17-27),
pinned by the reference's own test and by answers that follow from the
definition: DME(i, j) = sqrt(mean over atom pairs of (d_i - d_j)^2)."""
import numpy as np
import pytest

import oracle


def test_reference_test_identical_frames_give_zero():
    # test_pairwise_rmsd.py:64-75 (test_pairwise_rmsd_dme_zero_for_identical)
    c = np.array([[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]], [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]], np.float32)
    m32, _ = oracle.pairwise_dme(c)
    assert np.allclose(m32[0, 1], 0.0)


def test_two_atom_frames_give_distance_differences():
    # one atom pair: DME is |d_i - d_j|
    c = np.array([[[0, 0, 0], [1, 0, 0]], [[0, 0, 0], [2, 0, 0]], [[0, 0, 0], [0, 4, 0]], [[1, 1, 1], [1, 1, 1]]],
                 np.float32)
    m32, m64 = oracle.pairwise_dme(c)
    d = np.array([1.0, 2.0, 4.0, 0.0])
    np.testing.assert_array_equal(m64, np.abs(d[:, None] - d[None, :]))
    np.testing.assert_array_equal(m32, m64.astype(np.float32))


def test_three_atoms_known_answer():
    # triangle 3-4-5 against 6-8-10: pair distances (3, 4, 5) and (6, 8, 10)
    a = np.array([[0, 0, 0], [3, 0, 0], [0, 4, 0]], np.float32)
    c = np.stack([a, 2 * a])
    _, m64 = oracle.pairwise_dme(c)
    want = np.sqrt((9 + 16 + 25) / 3.0)
    assert m64[0, 1] == pytest.approx(want, rel=1e-15)
    assert m64[0, 0] == 0.0 and m64[1, 1] == 0.0 and m64[1, 0] == m64[0, 1]


def test_orthorhombic_minimum_image():
    # box 10: atoms 9 A apart along x are 1 A apart through the boundary;
    # a zero box length leaves that axis alone (apply_pbc's l > 0 test)
    c = np.array([[[0, 0, 0], [9, 0, 0]], [[0, 0, 0], [3, 0, 0]]], np.float32)
    _, m_none = oracle.pairwise_dme(c)
    _, m_box = oracle.pairwise_dme(c, box=[10, 10, 10])
    _, m_zero = oracle.pairwise_dme(c, box=[0, 10, 10])
    assert m_none[0, 1] == 6.0
    assert m_box[0, 1] == 2.0
    assert m_zero[0, 1] == 6.0
    # per-frame boxes: frame 1 in a box of 4 sees 3 A as 1 A
    _, m_pf = oracle.pairwise_dme(c, box=np.array([[10, 10, 10], [4, 4, 4]], np.float32))
    assert m_pf[0, 1] == 0.0


def test_small_selections_give_zeros():
    c = np.random.default_rng(0).normal(size=(5, 1, 3)).astype(np.float32)
    m32, m64 = oracle.pairwise_dme(c)
    assert (m32 == 0).all() and (m64 == 0).all()


def test_against_numpy_restatement():
    """A vectorised numpy statement of the same formula agrees to rounding
    (numpy sums in a different order)."""
    rng = np.random.default_rng(7)
    c = rng.normal(0, 5, size=(12, 17, 3)).astype(np.float32)
    box = np.array([7.5, 9.0, 11.0], np.float32)
    for b in (None, box):
        _, m64 = oracle.pairwise_dme(c, box=b)
        iu = np.triu_indices(c.shape[1], k=1)
        d = (c[:, iu[1], :] - c[:, iu[0], :]).astype(np.float64)  # f32 difference, widened
        if b is not None:
            L = b.astype(np.float64)
            q = d / L
            d = d - np.where(q >= 0, np.floor(q + 0.5), np.ceil(q - 0.5)) * L
        dist = np.sqrt((d ** 2).sum(-1))
        want = np.sqrt(((dist[:, None, :] - dist[None, :, :]) ** 2).mean(-1))
        np.testing.assert_allclose(m64, want, rtol=1e-12, atol=1e-12)
