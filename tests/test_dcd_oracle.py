"""The DCD oracle (oracle/dcd_oracle.py) against the reference reader's own
known answers (crates/traj-io/src/dcd.rs tests, 1142-1316) and against an
independent numpy decode of synthetic files in every record variant."""
import math
import struct

import numpy as np
import pytest

import dcd_files
import dcd_oracle as D


def _w(tmp_path, name, frames, **kw):
    p = tmp_path / name
    dcd_files.write(p, frames, **kw)
    return str(p)


def test_reject_invalid_header(tmp_path):
    p = tmp_path / "bad.dcd"
    p.write_bytes(bytes([1, 2, 3, 4]))
    with pytest.raises(D.DcdError) as e:
        D.DcdReader(str(p))
    assert e.value.kind in ("unsupported", "io", "parse")
    p.write_bytes(bytes(range(16)))
    with pytest.raises(D.DcdError) as e:
        D.DcdReader(str(p))
    assert e.value.kind == "unsupported"


def test_read_frame_without_unitcell_record(tmp_path):
    fr = np.array([[[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]], np.float32)
    r = D.DcdReader(_w(tmp_path, "no_box.dcd", fr))
    c, k, _ = r.read_chunk(1)
    assert r.header_frames == 1 and r.n_atoms == 2
    assert k[0] == 0
    np.testing.assert_array_equal(c[0], fr[0])


def test_read_frame_selected_endpoints_and_reset(tmp_path):
    fr = np.array([[[1, 10, 100], [2, 20, 200], [3, 30, 300], [4, 40, 400]]], np.float32)
    r = D.DcdReader(_w(tmp_path, "sel.dcd", fr))
    c, _, _ = r.read_chunk(1, selection=[3, 1])
    np.testing.assert_array_equal(c[0], [[4, 40, 400], [2, 20, 200]])
    r.reset()
    c, _, _ = r.read_chunk(1)
    np.testing.assert_array_equal(c[0], fr[0])
    with pytest.raises(D.DcdError) as e:
        r.reset()
        r.read_chunk(1, selection=[0, 4])
    assert e.value.kind == "mismatch" and "selection index 4 out of bounds" in e.value.msg


def test_skip_frames(tmp_path):
    fr = np.array([[[1, 2, 3]], [[4, 5, 6]], [[7, 8, 9]]], np.float32)
    r = D.DcdReader(_w(tmp_path, "skip.dcd", fr))
    assert r.skip_frames(2) == 2
    c, _, _ = r.read_chunk(1)
    np.testing.assert_array_equal(c[0], [[7, 8, 9]])
    assert r.read_chunk(5)[0].shape[0] == 0


def test_zero_unitcell_is_none_and_charmm_layout(tmp_path):
    fr = np.array([[[1, 2, 3]]], np.float32)
    r = D.DcdReader(_w(tmp_path, "zero.dcd", fr, cells=[[0.0] * 6]))
    c, k, _ = r.read_chunk(1)
    assert k[0] == 0
    np.testing.assert_array_equal(c[0], [[1, 2, 3]])
    # CHARMM order [A, gamma, B, beta, alpha, C], angles as cosines
    r = D.DcdReader(_w(tmp_path, "charmm.dcd", fr, cells=[[10.0, 0.0, 20.0, 0.0, 0.0, 30.0]], charmm_version=24))
    _, k, m = r.read_chunk(1)
    assert k[0] == 1
    np.testing.assert_array_equal(m[0].reshape(3, 3), np.diag([10.0, 20.0, 30.0]).astype(np.float32))


def test_triclinic_cell_matches_vectors(tmp_path):
    """The NAMD/VMD cosine convention (dcd.rs:1504-1536): A, cos(gamma), B,
    cos(beta), cos(alpha), C gives the box vectors of the reference's test."""
    a, b, c, al, be, ga = 10.0, 20.0, 30.0, 80.0, 70.0, 60.0
    cell = [a, math.cos(math.radians(ga)), b, math.cos(math.radians(be)), math.cos(math.radians(al)), c]
    fr = np.zeros((1, 3, 3), np.float32)
    r = D.DcdReader(_w(tmp_path, "tri.dcd", fr, cells=[cell], charmm_version=24))
    _, k, m = r.read_chunk(1)
    assert k[0] == 2
    gr, br, ar = (math.radians(x) for x in (ga, be, al))
    cx = c * math.cos(br)
    cy = c * (math.cos(ar) - math.cos(br) * math.cos(gr)) / math.sin(gr)
    want = [a, 0, 0, b * math.cos(gr), b * math.sin(gr), 0, cx, cy, math.sqrt(c * c - cx * cx - cy * cy)]
    np.testing.assert_allclose(m[0], want, rtol=1e-6, atol=1e-5)
    # degrees instead of cosines, standard layout
    r = D.DcdReader(_w(tmp_path, "deg.dcd", fr, cells=[[a, b, c, al, be, ga]]))
    _, k, m2 = r.read_chunk(1)
    assert k[0] == 2
    np.testing.assert_allclose(m2[0], want, rtol=1e-6, atol=1e-5)


def _numpy_decode(path, n_atoms, n_frames, endian, marker, cell_bytes, data_start):
    raw = np.fromfile(path, np.uint8)
    rec = 4 * n_atoms
    per = (2 * marker + cell_bytes if cell_bytes else 0) + 3 * (2 * marker + rec)
    out = np.empty((n_frames, n_atoms, 3), np.float32)
    for f in range(n_frames):
        x0 = data_start + f * per + (2 * marker + cell_bytes if cell_bytes else 0) + marker
        for c in range(3):
            o = x0 + c * (rec + 2 * marker)
            out[f, :, c] = raw[o:o + rec].view(endian + "f4")
    return out


@pytest.mark.parametrize("endian,marker,cell_bytes,header_len,titles", [
    ("<", 4, 0, 84, 1), (">", 4, 48, 84, 2), ("<", 8, 24, 164, 1), (">", 8, 0, 84, 3), ("<", 4, 48, 164, 0)])
def test_oracle_matches_numpy_decode(tmp_path, endian, marker, cell_bytes, header_len, titles):
    rng = np.random.default_rng(3)
    fr = rng.normal(0, 20, (7, 53, 3)).astype(np.float32)
    cells = [[30.0 + i, 40.0, 50.0, 90.0, 90.0, 90.0] for i in range(7)] if cell_bytes else None
    p = _w(tmp_path, "v.dcd", fr, cells=cells, endian=endian, marker=marker, cell_bytes=cell_bytes or 48,
           header_len=header_len, titles=titles)
    r = D.DcdReader(p, length_scale=0.5)
    c, k, m = r.read_chunk(100)
    np.testing.assert_array_equal(c, (_numpy_decode(p, 53, 7, endian, marker, cell_bytes, r.data_start)
                                      * np.float32(0.5)).astype(np.float32))
    if cell_bytes:
        assert np.all(k == 1)
        np.testing.assert_array_equal(m[:, 0], (np.float32(30.0) + np.arange(7, dtype=np.float32)) * np.float32(0.5))
    else:
        assert np.all(k == 0)


def test_damaged_files(tmp_path):
    fr = np.arange(4 * 5 * 3, dtype=np.float32).reshape(4, 5, 3)
    good = _w(tmp_path, "g.dcd", fr, cells=[[10.0, 10.0, 10.0, 90.0, 90.0, 90.0]] * 4)
    data = open(good, "rb").read()
    per = (8 + 48) + 3 * (8 + 20)
    start = len(data) - 4 * per
    # truncated inside the last frame: the first three read, the chunk reaching it fails with an IO error
    p = tmp_path / "trunc.dcd"
    p.write_bytes(data[:-10])
    r = D.DcdReader(str(p))
    assert r.read_chunk(3)[0].shape[0] == 3
    with pytest.raises(D.DcdError) as e:
        r.read_chunk(1)
    assert e.value.kind == "io"
    # end of file right after a unit cell: a clean end
    p.write_bytes(data + data[start:start + 56])
    assert D.read_all(str(p))[0].shape[0] == 4
    # a damaged end marker of frame 2's Y record
    bad = bytearray(data)
    off = start + 2 * per + 56 + 28 + 4 + 20
    bad[off:off + 4] = struct.pack("<I", 99)
    p.write_bytes(bytes(bad))
    r = D.DcdReader(str(p))
    assert r.read_chunk(2)[0].shape[0] == 2
    with pytest.raises(D.DcdError) as e:
        r.read_chunk(2)
    assert e.value.kind == "parse" and e.value.msg == "float record length mismatch"
    # frames of two layouts: the second frame carries no unit cell
    mixed = data[:start] + data[start:start + per] + data[start + per + 56:start + 2 * per]
    p.write_bytes(mixed)
    c, k, _ = D.read_all(str(p))
    np.testing.assert_array_equal(c, fr[:2])
    np.testing.assert_array_equal(k, [1, 0])
