"""DCD trajectories through the GPU decoder (Trajectory.open_dcd,
wmd_dcd_read, wmd_dcd_rmsd) against the oracle's sequential reader.

Parity is exact: coordinates, box kinds and box matrices are bit-identical to
the oracle's (the decoder only reorders bytes and multiplies by the length
scale in float32; unit cells use the same FP64 formulas and libm).  RMSD read
straight from a file agrees with the oracle's RMSD of the oracle-decoded
frames within 1e-5 A, the per-frame bar.
"""
import ctypes
import struct

import numpy as np
import pytest

import dcd_files
import dcd_oracle as D
import oracle
from warp_md import synth

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _system(n, positions0=None):
    import warp_md

    return warp_md.System.from_arrays({"name": ["CA" if i % 3 == 0 else "X" for i in range(n)],
                                       "resid": [i // 3 + 1 for i in range(n)]}, positions0=positions0)


def _write(tmp_path, name, frames, **kw):
    p = tmp_path / name
    dcd_files.write(p, frames, **kw)
    return str(p)


def _same_chunk(got, want_coords, want_kinds, want_mats):
    np.testing.assert_array_equal(got["coords"], want_coords)
    kinds = np.asarray(want_kinds)
    if np.any(kinds == 0):
        assert got["box"] is None and got["box_matrix"] is None
    else:
        np.testing.assert_array_equal(got["box_matrix"], want_mats.reshape(-1, 3, 3))
        if np.all(kinds == 1):
            np.testing.assert_array_equal(got["box"], want_mats[:, [0, 4, 8]])
        else:
            assert got["box"] is None


@pytest.mark.parametrize("endian,marker,cell_bytes,header_len,titles,title_pad,scale", [
    ("<", 4, 0, 84, 1, 0, None), (">", 4, 48, 84, 2, 0, 0.1), ("<", 8, 24, 164, 1, 0, None),
    (">", 8, 0, 84, 3, 0, 10.0), ("<", 4, 48, 164, 0, 2, None), (">", 8, 48, 84, 1, 1, 0.5)])
def test_read_chunks_match_oracle(tmp_path, endian, marker, cell_bytes, header_len, titles, title_pad, scale):
    import warp_md

    rng = np.random.default_rng(11)
    n, nf = 301, 23
    fr = rng.normal(0, 25, (nf, n, 3)).astype(np.float32)
    cells = None
    if cell_bytes:
        cells = [[30.0 + i, 0.0, 40.0, 0.0, 0.0, 50.0] if i % 3 else [31.0, 0.5, 41.0, 0.2, 0.1, 51.0]
                 for i in range(nf)]
    p = _write(tmp_path, "v.dcd", fr, cells=cells, endian=endian, marker=marker, cell_bytes=cell_bytes or 48,
               header_len=header_len, titles=titles, title_pad=title_pad, charmm_version=24 if cell_bytes else 0)
    system = _system(n)
    traj = warp_md.Trajectory.open_dcd(p, system, length_scale=scale)
    assert traj.n_frames() == nf and traj.n_atoms() == n and traj.n_frames_hint() == nf
    ref = D.DcdReader(p, 1.0 if scale is None else scale)
    for max_frames, sel in ((5, None), (7, [300, 0, 5, 5, 17]), (100, None)):
        got = traj.read_chunk(max_frames=max_frames, atom_indices=sel)
        want = ref.read_chunk(max_frames, selection=sel)
        _same_chunk(got, *want)
    assert traj.read_chunk() is None
    traj.reset()
    np.testing.assert_array_equal(traj.coords, D.read_all(p, 1.0 if scale is None else scale)[0])
    got = traj.read_frames([-1, 0, 4])
    np.testing.assert_array_equal(got["coords"], traj.coords[[nf - 1, 0, 4]])
    dev = traj.read_device(3, 9, atom_indices=[7, 2])
    np.testing.assert_array_equal(dev.cpu().numpy(), traj.coords[3:12][:, [7, 2]])
    traj.close()


def test_damaged_and_mixed_files(tmp_path):
    import warp_md

    fr = np.arange(4 * 5 * 3, dtype=np.float32).reshape(4, 5, 3)
    good = _write(tmp_path, "g.dcd", fr, cells=[[10.0, 10.0, 10.0, 90.0, 90.0, 90.0]] * 4)
    data = open(good, "rb").read()
    per = (8 + 48) + 3 * (8 + 20)
    start = len(data) - 4 * per
    system = _system(5)
    p = tmp_path / "d.dcd"
    # truncated inside the last frame: three frames read; the chunk that reaches the fourth fails (IO)
    p.write_bytes(data[:-10])
    t = warp_md.Trajectory.open_dcd(str(p), system)
    assert t.n_frames() == 3
    assert t.read_chunk(max_frames=3)["frames"] == 3
    with pytest.raises(warp_md.WarpMdError) as e:
        t.read_chunk(max_frames=1)
    assert e.value.code == -8 and str(e.value).startswith("io error")
    t.close()
    # end of file right after a unit cell: a clean end
    p.write_bytes(data + data[start:start + 56])
    t = warp_md.Trajectory.open_dcd(str(p), system)
    np.testing.assert_array_equal(t.coords, fr)
    t.close()
    # a damaged end marker in frame 2 that the open-time checks do not see:
    # the decoder finds it, frames 0-1 stay readable, a read reaching frame 2 fails (parse)
    bad = bytearray(data)
    off = start + 2 * per + 56 + 28 + 4 + 20
    bad[off:off + 4] = struct.pack("<I", 99)
    p.write_bytes(bytes(bad))
    t = warp_md.Trajectory.open_dcd(str(p), system)
    with pytest.raises(warp_md.WarpMdError) as e:
        t.read_chunk(max_frames=4)
    assert e.value.code == -9 and "float record length mismatch" in str(e.value)
    assert t.n_frames() == 2
    t.reset()
    np.testing.assert_array_equal(t.read_chunk(max_frames=2)["coords"], fr[:2])
    t.close()
    # frames of two layouts (the second has no unit cell): indexed frame by frame
    p.write_bytes(data[:start] + data[start:start + per] + data[start + per + 56:start + 2 * per]
                  + data[start + 2 * per:])
    t = warp_md.Trajectory.open_dcd(str(p), system)
    want = D.read_all(str(p))
    got = t.read_chunk(max_frames=10)
    np.testing.assert_array_equal(got["coords"], want[0])
    assert got["box"] is None
    t.close()
    # errors at open
    with pytest.raises(warp_md.WarpMdError) as e:
        warp_md.Trajectory.open_dcd(str(tmp_path / "missing.dcd"), system)
    assert e.value.code == -8
    p.write_bytes(bytes(range(16)))
    with pytest.raises(warp_md.WarpMdError) as e:
        warp_md.Trajectory.open_dcd(str(p), system)
    assert e.value.code == -5
    with pytest.raises(RuntimeError, match="atom count does not match"):
        warp_md.Trajectory.open_dcd(good, _system(6))
    t = warp_md.Trajectory.open_dcd(good, system)
    with pytest.raises(warp_md.WarpMdError, match="selection index 5 out of bounds"):
        t.read_chunk(atom_indices=[0, 5])
    t.close()


def test_rmsd_plan_from_dcd_matches_oracle(tmp_path):
    """RmsdPlan on an open DCD (wmd_dcd_rmsd: pread, copy, decode and RMSD
    kernels overlapped across 64 MiB batches) against the oracle."""
    import warp_md

    n, nf = 30_000, 420  # 360 KB frames: several batches
    fr, ref = synth.make_trajectory(n, nf, (0.05, 2.0), 21)
    p = _write(tmp_path, "big.dcd", fr, cells=[[80.0, 80.0, 80.0, 90.0, 90.0, 90.0]] * nf)
    system = _system(n, positions0=ref)
    for expr in ("all", "name CA"):
        sel = system.select(expr)
        idx = sel.as_array()
        for mode, r in (("topology", ref[idx]), ("frame0", fr[0][idx])):
            for align in (True, False):
                traj = warp_md.Trajectory.open_dcd(p, system)
                got = warp_md.RmsdPlan(sel, reference=mode, align=align).run(traj, system, dtype=np.float64)
                want = oracle.rmsd_frames(fr, r, selection=None if expr == "all" else idx, align=align)[1]
                assert got.shape == (nf,)
                np.testing.assert_allclose(got, want, rtol=0, atol=1e-5, err_msg=f"{expr} {mode} {align}")
                # the run consumed the trajectory
                assert warp_md.RmsdPlan(sel, reference=mode, align=align).run(traj, system).size == 0
                traj.close()


def test_dcd_rmsd_device_output_and_offsets(tmp_path, gpu_ctx):
    from warp_md import _native as N

    n, nf = 4000, 60
    fr, ref = synth.make_trajectory(n, nf, 0.7, 5)
    p = _write(tmp_path, "o.dcd", fr, endian=">", marker=8)
    ctx = gpu_ctx
    h = ctypes.c_void_p()
    ctx.check(ctx.lib.wmd_dcd_open(ctx.handle, p.encode(), 1.0, ctypes.byref(h)))
    try:
        sel = np.arange(5, n, 7, dtype=np.uint32)
        r = N.Reference.from_numpy(ctx, ref[sel])
        out = torch.zeros(nf, dtype=torch.float64, device="cuda")
        got = ctypes.c_int64()
        ctx.check(ctx.lib.wmd_dcd_rmsd(ctx.handle, h, 10, 1000, sel.ctypes.data, sel.size, r.handle, 1,
                                       out.data_ptr(), ctypes.byref(got), torch.cuda.current_stream().cuda_stream))
        assert got.value == nf - 10
        want = oracle.rmsd_frames(fr[10:], ref[sel], selection=sel)[1]
        np.testing.assert_allclose(out[: nf - 10].cpu().numpy(), want, rtol=0, atol=1e-5)
        r.close()
    finally:
        ctx.lib.wmd_dcd_close(ctx.handle, h)


def test_dcd_boxes_feed_dme_pbc(tmp_path):
    """A DCD with orthorhombic unit cells exposes per-frame box lengths
    (Trajectory.box, bit-identical to the oracle reader's), and
    PairwiseRmsdPlan(metric="dme", pbc="orthorhombic") uses them; a file
    without cells has no box and the PBC form stops with the reference's
    mismatch."""
    import warp_md

    rng = np.random.default_rng(4)
    n, nf = 40, 19
    fr = rng.uniform(0, 20, (nf, n, 3)).astype(np.float32)
    cells = [[20.0 + 0.1 * i, 0.0, 19.0, 0.0, 0.0, 21.0 - 0.05 * i] for i in range(nf)]  # CHARMM: A, cos g, B, cos b, cos a, C
    p = _write(tmp_path, "cells.dcd", fr, cells=cells, charmm_version=24)
    coords, kinds, mats = D.read_all(p)
    assert np.all(np.asarray(kinds) == 1)
    want_box = np.asarray(mats)[:, [0, 4, 8]]
    system = _system(n)
    sel = system.select("name CA")
    idx = sel.as_array()
    traj = warp_md.Trajectory.open_dcd(p, system)
    np.testing.assert_array_equal(traj.box, want_box)
    got = warp_md.PairwiseRmsdPlan(sel, metric="dme", pbc="orthorhombic").run(traj, system)
    np.testing.assert_array_equal(got, oracle.pairwise_dme(np.asarray(coords)[:, idx], box=want_box)[0])
    traj.close()
    q = _write(tmp_path, "nocells.dcd", fr)
    traj = warp_md.Trajectory.open_dcd(q, system)
    assert traj.box is None
    with pytest.raises(warp_md.WarpMdError, match="orthorhombic box required"):
        warp_md.PairwiseRmsdPlan(sel, metric="dme", pbc="orthorhombic").run(traj, system)
    traj.close()
