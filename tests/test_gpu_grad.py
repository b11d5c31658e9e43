"""dRMSD/dx from the hand-written backward kernel (torch.autograd.Function)
against the oracle's analytic FP64 gradient and FP64 central differences.

The reference has no gradient, so these are the pins: the analytic formula of
the oracle (itself checked by central differences in test_oracle.py) and
central differences of the FP64 RMSD with h = 1e-4 A on random atoms.
Tolerance: |g_gpu - g_fp64| <= 1e-5 * max|g| + 1e-7 (the result is float32).
"""
import numpy as np
import pytest

import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _fp64_rmsd(x, y):
    xc = x - x.mean(0)
    yc = y - y.mean(0)
    u, s, vt = np.linalg.svd(xc.T @ yc)
    d = np.sign(np.linalg.det(vt.T @ u.T))
    msd = ((xc ** 2).sum() + (yc ** 2).sum() - 2 * (s[0] + s[1] + d * s[2])) / len(x)
    return np.sqrt(max(msd, 0.0))


def _check(g_gpu, g_ref):
    tol = 1e-5 * np.abs(g_ref).max() + 1e-7
    err = np.abs(g_gpu - g_ref).max()
    assert err <= tol, (err, tol)


def test_backward_matches_analytic_small():
    from warp_md.torch_ops import rmsd

    for n, F, seed in [(3, 4, 1), (50, 8, 2), (1024, 5, 3), (2049, 6, 4), (5000, 3, 5)]:
        fr, ref = synth.make_trajectory(n, F, 0.3, seed)
        x = torch.from_numpy(fr).cuda().requires_grad_(True)
        y = torch.from_numpy(ref).cuda()
        val = rmsd(x, y)
        val.sum().backward()
        rm, g = oracle.rmsd_grad(fr, ref)
        np.testing.assert_allclose(val.detach().cpu().numpy(), rm, atol=1e-5)
        _check(x.grad.cpu().numpy(), g)


def test_backward_weighted_upstream_and_selection():
    from warp_md.torch_ops import rmsd

    fr, _ = synth.make_trajectory(600, 10, 0.3, 7)
    sel = np.arange(0, 600, 3)
    # a reference that is none of the frames: the gradient of |.| at RMSD 0 is undefined
    ref = (fr[0][sel] + np.random.default_rng(1).normal(0, 0.3, (sel.size, 3))).astype(np.float32)
    x = torch.from_numpy(fr).cuda().requires_grad_(True)
    w = torch.linspace(-1, 2, 10, device="cuda", dtype=torch.float64)
    val = rmsd(x, torch.from_numpy(ref).cuda(), torch.from_numpy(sel.astype(np.int32)).cuda())
    (val * w).sum().backward()
    rm, g = oracle.rmsd_grad(fr, ref, selection=sel)
    g = g * w.cpu().numpy()[:, None, None]
    got = x.grad.cpu().numpy()
    _check(got, g)
    mask = np.ones(600, bool)
    mask[sel] = False
    assert np.all(got[:, mask] == 0)


def test_differentiable_workload_with_finite_differences():
    """4,096 frames x 2,000 atoms, sigma = 0.3 A: every gradient against the
    analytic FP64 gradient; FP64 central differences (h = 1e-4 A) on 64 random
    atoms of 8 frames."""
    from warp_md.torch_ops import rmsd

    fr, ref = synth.make_trajectory(2000, 4096, 0.3, seed=2)
    x = torch.from_numpy(fr).cuda().requires_grad_(True)
    val = rmsd(x, torch.from_numpy(ref).cuda())
    val.sum().backward()
    got = x.grad.cpu().numpy()
    rm, g = oracle.rmsd_grad(fr, ref)
    np.testing.assert_allclose(val.detach().cpu().numpy(), rm, atol=1e-5)
    _check(got, g)
    rng = np.random.default_rng(0)
    h = 1e-4
    y64 = ref.astype(np.float64)
    for f in rng.choice(4096, 8, replace=False):
        x64 = fr[f].astype(np.float64)
        for atom in rng.choice(2000, 64, replace=False):
            for c in range(3):
                xp = x64.copy(); xp[atom, c] += h
                xm = x64.copy(); xm[atom, c] -= h
                fd = (_fp64_rmsd(xp, y64) - _fp64_rmsd(xm, y64)) / (2 * h)
                assert abs(fd - got[f, atom, c]) < 1e-6 + 1e-4 * abs(fd), (f, atom, c, fd, got[f, atom, c])


def test_zero_rmsd_gives_zero_gradient():
    from warp_md.torch_ops import rmsd

    _, ref = synth.make_trajectory(30, 1, 0.0, 3)
    x = torch.from_numpy(np.stack([ref, ref])).cuda().requires_grad_(True)
    val = rmsd(x, torch.from_numpy(ref).cuda())
    val.sum().backward()
    assert torch.all(val < 1e-5)
    assert torch.all(torch.isfinite(x.grad))


def test_gradient_buffer_fully_written():
    """Without a selection the gradient buffer is not zero-filled first: the
    kernel must write every element.  Freed NaN blocks of the same size are
    left in torch's caching allocator so that unwritten entries would show;
    a dense prefix (reference shorter than the frame) still gets zeros beyond
    it, and a selection gets zeros outside it."""
    from warp_md.torch_ops import rmsd

    for n, F, seed in [(1000, 7, 11), (2048, 4, 12), (37, 9, 13)]:
        fr, ref = synth.make_trajectory(n, F, 0.3, seed)
        for _ in range(4):
            junk = torch.full((F, n, 3), float("nan"), device="cuda")
            del junk
        x = torch.from_numpy(fr).cuda().requires_grad_(True)
        rmsd(x, torch.from_numpy(ref).cuda()).sum().backward()
        g = x.grad.cpu().numpy()
        assert np.isfinite(g).all()
        _check(g, oracle.rmsd_grad(fr, ref)[1])
        # dense prefix: atoms past the reference get a zero gradient
        k = n // 2
        for _ in range(4):
            junk = torch.full((F, n, 3), float("nan"), device="cuda")
            del junk
        x2 = torch.from_numpy(fr).cuda().requires_grad_(True)
        rmsd(x2, torch.from_numpy(np.ascontiguousarray(ref[:k])).cuda()).sum().backward()
        g2 = x2.grad.cpu().numpy()
        assert np.isfinite(g2).all()
        assert (g2[:, k:] == 0).all()
        _check(g2[:, :k], oracle.rmsd_grad(np.ascontiguousarray(fr[:, :k]), ref[:k])[1])
