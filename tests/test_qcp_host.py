"""The library's QCP header (warp-md_b200/csrc/qcp.cuh) compiled for the host
and checked against the oracle's SVD route: lambda_max, the degenerate-root
fallback, and the rotation convention (R maps frame coordinates onto the
reference, as R = V U^T in plan.rs:1214-1221).  The mixed-precision MSD of the
tensor-core pairwise epilogue is checked against the FP64 route on the same
exact integer sums."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def qlib(tmp_path_factory):
    out = tmp_path_factory.mktemp("qcp") / "libqcp_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(REPO, "warp-md_b200", "csrc"),
                    os.path.join(HERE, "native", "qcp_host.cpp"), "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.t_qcp_lambda.argtypes = [dp, ctypes.c_double, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.t_qcp_lambda.restype = ctypes.c_double
    L.t_lambda_svd.argtypes = [dp]
    L.t_lambda_svd.restype = ctypes.c_double
    L.t_rotation_qcp.argtypes = [dp, ctypes.c_double, dp]
    L.t_rotation_svd.argtypes = [dp, dp]
    ip = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
    L.t_qcp_msd_mixed.argtypes = [ip, ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_float,
                                  ctypes.POINTER(ctypes.c_float)]
    L.t_qcp_msd_mixed.restype = ctypes.c_int
    return L


def _h_and_g(x, y):
    xc = x - x.mean(0)
    yc = y - y.mean(0)
    return np.ascontiguousarray(xc.T @ yc), (xc ** 2).sum(), (yc ** 2).sum()


def _lam(qlib, h, e0):
    it, fb = ctypes.c_int(), ctypes.c_int()
    return qlib.t_qcp_lambda(h.reshape(9), e0, ctypes.byref(it), ctypes.byref(fb)), it.value, fb.value


def test_lambda_matches_svd_random(qlib):
    from warp_md import synth

    rng = np.random.default_rng(5)
    for trial in range(50):
        n = int(rng.integers(3, 300))
        fr, ref = synth.make_trajectory(n, 1, float(rng.uniform(0.01, 3)), trial)
        x, y = fr[0].astype(np.float64), ref.astype(np.float64)
        h, gx, gy = _h_and_g(x, y)
        lam, it, fb = _lam(qlib, h, 0.5 * (gx + gy))
        r, ss = oracle.kabsch_rotation(h)
        assert abs(lam - ss) <= 1e-12 * max(1.0, ss), (trial, lam, ss)
        assert it < 60


def test_degenerate_roots_fall_back(qlib):
    # collinear: H rank 1 -> lambda_max is a double root of the quartic
    x = np.zeros((10, 3)); x[:, 0] = np.arange(10.0)
    y = x @ np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1.0]]).T
    h, gx, gy = _h_and_g(x, y)
    lam, it, fb = _lam(qlib, h, 0.5 * (gx + gy))
    assert fb == 1
    assert abs(lam - 0.5 * (gx + gy)) < 1e-9 * gx
    # identical planar structure: double root again
    p = np.zeros((12, 3)); p[:, :2] = np.random.default_rng(2).normal(size=(12, 2))
    h, gx, gy = _h_and_g(p, p)
    lam, it, fb = _lam(qlib, h, 0.5 * (gx + gy))
    assert abs(lam - gx) < 1e-12 * gx
    # all atoms at one point: lambda 0
    z = np.ones((5, 3))
    h, gx, gy = _h_and_g(z, z)
    lam, it, fb = _lam(qlib, h, 0.5 * (gx + gy))
    assert lam == 0.0


def test_rotation_matches_kabsch(qlib):
    rng = np.random.default_rng(9)
    from warp_md import synth

    for trial in range(30):
        fr, ref = synth.make_trajectory(int(rng.integers(4, 200)), 1, 0.3, 100 + trial)
        x, y = fr[0].astype(np.float64), ref.astype(np.float64)
        h, gx, gy = _h_and_g(x, y)
        lam, _, _ = _lam(qlib, h, 0.5 * (gx + gy))
        r = np.empty(9)
        qlib.t_rotation_qcp(h.reshape(9), lam, r)
        r_ref, _ = oracle.kabsch_rotation(h)
        np.testing.assert_allclose(r.reshape(3, 3), r_ref, atol=1e-9)
        rs = np.empty(9)
        qlib.t_rotation_svd(h.reshape(9), rs)
        np.testing.assert_allclose(rs.reshape(3, 3), r_ref, atol=1e-9)


def test_mirror_uses_reflection_fix(qlib):
    from warp_md import synth

    fr, ref = synth.make_trajectory(30, 1, 0.05, 4)
    x = fr[0].astype(np.float64).copy()
    x[:, 2] *= -1
    h, gx, gy = _h_and_g(x, ref.astype(np.float64))
    assert np.linalg.det(h) < 0
    lam, _, _ = _lam(qlib, h, 0.5 * (gx + gy))
    _, ss = oracle.kabsch_rotation(h)
    assert abs(lam - ss) < 1e-10 * ss


def _random_rotation(rng):
    q = rng.normal(size=4)
    w, a, b, c = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)],
                     [2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)],
                     [2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)]])


def test_mixed_precision_msd_matches_fp64_route(qlib):
    """qcp_msd_mixed (the tensor-core epilogue's QCP: FP64 only for det(D I - 2K),
    FP32 for the other coefficients and Newton) against qcp_lambda in FP64 on
    the same exact integer sums.  Inputs as the i8 limb path builds them:
    centred coordinates quantised to steps s of 6e-6 .. 4.2e-5 A, H and the
    self-sums exact in units of s^2.  Accepted roots agree within 5e-6 A of
    RMSD; collinear and nearly collinear structures are handed back to the
    FP64 route."""
    rng = np.random.default_rng(11)
    worst = 0.0
    handed_back = {"general": 0, "collinear": 0}
    counts = {"general": 0, "collinear": 0}
    for trial in range(400):
        n = int(rng.integers(3, 1500))
        kind = ("general", "general", "planar", "collinear")[trial % 4]
        sig = 10 ** rng.uniform(-3.5, 0.5)
        s = 6e-6 * (1 + trial % 7)
        x = 15 * rng.normal(size=(n, 3))
        if kind == "planar":
            x[:, 2] = 0.0
        if kind == "collinear":
            x[:, 1] = (trial % 8 == 3) * 1e-3 * rng.normal(size=n)
            x[:, 2] = 0.0
        y = x @ _random_rotation(rng).T + sig * rng.normal(size=(n, 3))
        qx = np.rint((x - x.mean(0)) / s).astype(np.int64)
        qy = np.rint((y - y.mean(0)) / s).astype(np.int64)
        h = np.ascontiguousarray((qx.T @ qy).reshape(9))
        gx, gy = float((qx * qx).sum()), float((qy * qy).sum())
        lam, _, _ = _lam(qlib, h.astype(np.float64).reshape(3, 3), 0.5 * (gx + gy))
        ref = np.sqrt(max(gx + gy - 2 * lam, 0.0) / n * s * s)
        m = ctypes.c_float()
        ok = qlib.t_qcp_msd_mixed(h, gx, gy, float(n), float(s * s), ctypes.byref(m))
        group = "collinear" if kind == "collinear" else "general"
        counts[group] += 1
        if not ok:
            handed_back[group] += 1
            continue
        err = abs(np.sqrt(m.value) - ref)
        worst = max(worst, err)
        assert err <= 5e-6, (trial, kind, n, sig, np.sqrt(m.value), ref)
    assert worst <= 5e-6
    # general and planar structures stay on the mixed route; exactly collinear ones do not
    assert handed_back["general"] <= counts["general"] // 50, handed_back
    assert handed_back["collinear"] >= counts["collinear"] // 4, handed_back

