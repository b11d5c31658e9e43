"""Writes DCD files for the reader tests: little or big endian, 4- or 8-byte
record markers, optional unit-cell records (f64 or f32), CHARMM version slot,
and damaged variants.  The record structure is the one warp-md's reader
expects (crates/traj-io/src/dcd.rs) and its own test writer produces
(write_test_dcd_multi, dcd.rs:1382-1428)."""
from __future__ import annotations

import struct
from typing import Optional, Sequence

import numpy as np


def record(payload: bytes, endian: str = "<", marker: int = 4, length: Optional[int] = None,
           end_length: Optional[int] = None) -> bytes:
    fmt = endian + ("I" if marker == 4 else "Q")
    n = len(payload) if length is None else length
    e = n if end_length is None else end_length
    return struct.pack(fmt, n) + payload + struct.pack(fmt, e)


def header(n_atoms: int, n_frames: int, endian: str = "<", marker: int = 4, cell_flag: bool = False,
           charmm_version: int = 0, header_len: int = 84, titles: int = 1, title: bytes = b"WARP_MD_B200_TEST",
           title_pad: int = 0) -> bytes:
    icntrl = [0] * 20
    icntrl[0] = n_frames
    icntrl[10] = 1 if cell_flag else 0
    icntrl[19] = charmm_version
    hdr = b"CORD" + struct.pack(endian + "20i", *icntrl)
    hdr += b"\0" * (header_len - len(hdr))
    line = title.ljust(80, b" ")[:80]
    tit = struct.pack(endian + "i", titles) + line * titles + b" " * title_pad
    return (record(hdr, endian, marker) + record(tit, endian, marker)
            + record(struct.pack(endian + "i", n_atoms), endian, marker))


def frame(xyz: np.ndarray, cell: Optional[Sequence[float]] = None, endian: str = "<", marker: int = 4,
          cell_bytes: int = 48) -> bytes:
    out = b""
    if cell is not None:
        dt = endian + ("f8" if cell_bytes == 48 else "f4")
        out += record(np.asarray(cell, dt).tobytes(), endian, marker)
    for c in range(3):
        out += record(np.ascontiguousarray(xyz[:, c], endian + "f4").tobytes(), endian, marker)
    return out


def write(path, frames: np.ndarray, cells=None, endian: str = "<", marker: int = 4, cell_bytes: int = 48,
          charmm_version: int = 0, header_len: int = 84, titles: int = 1, header_frames: Optional[int] = None,
          tail: bytes = b"", title_pad: int = 0) -> None:
    """frames [F][N][3]; cells None, or a per-frame list of 6 values / None;
    title_pad extra bytes in the title record (records off 4-byte alignment)."""
    frames = np.asarray(frames, np.float32)
    f_, n = frames.shape[0], frames.shape[1]
    has_cell = cells is not None and any(c is not None for c in cells)
    parts = [header(n, f_ if header_frames is None else header_frames, endian, marker, has_cell, charmm_version,
                    header_len, titles, title_pad=title_pad)]
    for i in range(f_):
        parts.append(frame(frames[i], None if cells is None else cells[i], endian, marker, cell_bytes))
    parts.append(tail)
    with open(path, "wb") as fh:
        fh.write(b"".join(parts))
