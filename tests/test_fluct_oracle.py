"""Fluctuations and per-residue RMSD in the oracle, and the host-side
aggregation of the fluct wrappers, on the CPU.

Pins: the known answers of the reference's test_fluct.py (an atom moving
0, 1, 2 along x has RMSF sqrt(2/3) and u_xx = 2/3; the frame subset [2, 0]
gives RMSF 1), numpy's variance/covariance for random data, and an
independent numpy restatement of RmsdPerResPlan's CPU path (rms.rs:633-671).
"""
import numpy as np

import oracle


def _ref_test_coords():
    c = np.zeros((3, 4, 3), np.float32)
    c[:, 1, 0] = [0.0, 1.0, 2.0]
    c[:, 3, 0] = [2.0, 3.0, 4.0]
    return c


def test_known_answers_from_reference_tests():
    c = _ref_test_coords()
    r, a = oracle.rmsf(c)
    r0 = np.sqrt(2.0 / 3.0)
    np.testing.assert_allclose(r, [0.0, r0, 0.0, r0], rtol=1e-12)
    np.testing.assert_allclose(a[[1, 3], 0], [2.0 / 3.0, 2.0 / 3.0], rtol=1e-12)
    np.testing.assert_allclose(a[[0, 2]], 0.0, atol=1e-15)
    np.testing.assert_allclose(a[:, 1:], 0.0, atol=1e-15)
    r, a = oracle.rmsf(c[[2, 0]])
    np.testing.assert_allclose(r, [0.0, 1.0, 0.0, 1.0], rtol=1e-12)
    np.testing.assert_allclose(a[[1, 3], 0], [1.0, 1.0], rtol=1e-12)


def test_rmsf_and_adp_against_numpy():
    rng = np.random.default_rng(1)
    c = (rng.normal(0, 0.7, (50, 30, 3)) + rng.uniform(-300, 300, (1, 30, 3))).astype(np.float32)
    sel = np.array([0, 3, 7, 29, 12], np.uint32)
    r, a = oracle.rmsf(c, selection=sel)
    x = c[:, sel].astype(np.float64)
    np.testing.assert_allclose(r, np.sqrt(x.var(axis=0).sum(axis=1)), rtol=1e-9)
    cov = np.einsum("fia,fib->iab", x - x.mean(0), x - x.mean(0)) / x.shape[0]
    want = np.stack([cov[:, 0, 0], cov[:, 1, 1], cov[:, 2, 2], cov[:, 0, 1], cov[:, 0, 2], cov[:, 1, 2]], axis=1)
    np.testing.assert_allclose(a, want, rtol=1e-6, atol=1e-9)


def _numpy_perres(c, ref_all, groups, sel, align):
    out = np.zeros((c.shape[0], len(groups)))
    for f in range(c.shape[0]):
        x = c[f].astype(np.float64)
        y = ref_all.astype(np.float64)
        if align:
            cx, cy = x[sel].mean(0), y[sel].mean(0)
            h = (x[sel] - cx).T @ (y[sel] - cy)
            u, _s, vt = np.linalg.svd(h)
            r = vt.T @ u.T
            if np.linalg.det(r) < 0:
                vt[-1] *= -1
                r = vt.T @ u.T
            moved, target = (x - cx) @ r.T, y - cy
        else:
            moved, target = x, y
        for g, atoms in enumerate(groups):
            d = moved[atoms] - target[atoms]
            out[f, g] = np.sqrt((d * d).sum() / max(1, len(atoms)))
    return out


def test_perres_against_numpy():
    from warp_md import synth

    fr, ref = synth.make_trajectory(60, 5, 0.5, 9)
    rng = np.random.default_rng(2)
    resid = np.sort(rng.integers(0, 12, 60))
    sel = np.arange(0, 60, 2)
    groups = [sel[resid[sel] == r] for r in np.unique(resid[sel])] + [np.zeros(0, np.int64)]
    for align in (True, False):
        got = oracle.rmsd_perres(fr, ref, groups, selection=sel, align=align)
        np.testing.assert_allclose(got, _numpy_perres(fr, ref, groups, sel, align), rtol=0, atol=1e-10)


def test_fluct_aggregation_modes():
    """test_fluct_aggregate_fallback_modes of the reference (python/warp_md/tests/test_fluct.py)."""
    from warp_md.analysis.fluct import _aggregate

    class _Sys:
        def atom_table(self):
            return {"resid": [1, 1, 2, 2]}

    values = np.array([1.0, 3.0, 5.0, 7.0], dtype=np.float32)
    indices = np.array([0, 1, 2, 3], dtype=np.int64)
    np.testing.assert_allclose(_aggregate(values, indices, _Sys(), False, False),
                               np.array([[0.0, 1.0], [1.0, 3.0], [2.0, 5.0], [3.0, 7.0]], dtype=np.float32))
    np.testing.assert_allclose(_aggregate(values, indices, _Sys(), True, False),
                               np.array([[1.0, 2.0], [2.0, 6.0]], dtype=np.float32))
    np.testing.assert_allclose(_aggregate(values, indices, _Sys(), False, True),
                               np.array([[0.0, 4.0]], dtype=np.float32))
