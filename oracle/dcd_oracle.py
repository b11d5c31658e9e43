"""Sequential DCD reader: a plain restatement of warp-md's DcdReader.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and the CPU legs of
``bench.py`` as the checker for the GPU decoder; the product never imports it.

Follows crates/traj-io/src/dcd.rs record by record:
  * open: detect_header_marker (833-858; 8-byte markers tried first, then 4;
    header record length 84 or 164), header trailer check (45-57),
    parse_n_frames (1103-1117), parse_unitcell_layout (1119-1135; CHARMM
    version > 0 -> [A, gamma, B, beta, alpha, C]), title record skip (61),
    natoms record (63-76);
  * read_frame (207-291) / read_frame_selected_cached (293-381): an optional
    unit-cell record of 24 (f32) or 48 (f64) bytes, then X, Y, Z records of
    n_atoms floats, every end marker checked; end of file before a frame's
    first marker (or right after its unit cell) ends the trajectory, anywhere
    else it is an IO error;
  * read_unitcell_with_len (978-1022) and box_from_values (1024-1093) with the
    alternate-layout fallback; coordinates times length_scale in float32.

Errors carry the reference's TrajError kind ("io", "parse", "unsupported",
"mismatch") and message.
"""
from __future__ import annotations

import math
import struct
from typing import List, Optional, Sequence, Tuple

import numpy as np


class DcdError(Exception):
    def __init__(self, kind: str, msg: str):
        super().__init__(f"{kind}: {msg}")
        self.kind = kind
        self.msg = msg


# Box kinds: 0 = none, 1 = orthorhombic, 2 = triclinic; m = a, b, c rows.
Box = Tuple[int, np.ndarray]


def _none_box() -> Box:
    return 0, np.zeros(9, np.float32)


def _to_radians(v: float) -> float:
    return v * (math.pi / 180.0)


def _angle_to_radians(v: float) -> float:
    """unitcell_angle_to_radians (dcd.rs:1095-1101): cosines when |v| <= 1."""
    if abs(v) <= 1.0:
        return math.acos(min(max(v, -1.0), 1.0))
    return _to_radians(v)


def box_from_values(values: Sequence[float], charmm: bool, length_scale: float) -> Box:
    """box_from_values (dcd.rs:1024-1093), FP64 then float32."""
    v = [float(x) for x in values]
    if charmm:
        a, b, c, al, be, ga = v[0], v[2], v[5], v[4], v[3], v[1]
    else:
        a, b, c, al, be, ga = v
    s = float(np.float32(length_scale))
    a *= s
    b *= s
    c *= s
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)) or a <= 1e-6 or b <= 1e-6 or c <= 1e-6:
        return _none_box()
    ar, br, gr = _angle_to_radians(al), _angle_to_radians(be), _angle_to_radians(ga)
    if not (math.isfinite(ar) and math.isfinite(br) and math.isfinite(gr)):
        return _none_box()
    ninety = math.pi / 2
    if abs(ar - ninety) < 1e-3 and abs(br - ninety) < 1e-3 and abs(gr - ninety) < 1e-3:
        m = np.zeros(9, np.float32)
        m[0], m[4], m[8] = a, b, c
        return 1, m
    ca, cb, cg, sg = math.cos(ar), math.cos(br), math.cos(gr), math.sin(gr)
    if abs(sg) < 1e-8:
        return _none_box()
    cx = c * cb
    cy = c * (ca - cb * cg) / sg
    cz2 = c * c - cx * cx - cy * cy
    if not math.isfinite(cz2) or cz2 <= 0.0:
        return _none_box()
    m = np.array([a, 0.0, 0.0, b * cg, b * sg, 0.0, cx, cy, math.sqrt(cz2)], np.float64).astype(np.float32)
    return 2, m


class DcdReader:
    """The reference reader over an in-memory copy of the file (test sizes)."""

    def __init__(self, path: str, length_scale: float = 1.0):
        try:
            with open(path, "rb") as fh:
                self.data = fh.read()
        except OSError as e:
            raise DcdError("io", str(e)) from None
        self.pos = 0
        self.scale = np.float32(length_scale)
        self._detect()
        hlen = self.header_len
        header = self._read_exact(hlen)
        if self._marker() != hlen:
            raise DcdError("parse", "DCD header record length mismatch")
        self.header_frames = None
        if header[0:4] == b"CORD":
            n = struct.unpack(self.e + "i", header[4:8])[0]
            self.header_frames = n if n > 0 else None
        self.charmm = len(header) >= 84 and struct.unpack(self.e + "i", header[80:84])[0] > 0
        self._skip_record(self._marker())
        if self._marker() != 4:
            raise DcdError("parse", "unexpected natoms record length")
        natoms = struct.unpack(self.e + "i", self._read_exact(4))[0]
        if self._marker() != 4:
            raise DcdError("parse", "natoms record length mismatch")
        if natoms <= 0:
            raise DcdError("parse", "invalid natoms")
        self.n_atoms = natoms
        self.data_start = self.pos

    # -- records ---------------------------------------------------------
    def _detect(self):
        if len(self.data) < 8:
            raise DcdError("io", "failed to fill whole buffer")
        le8, be8 = struct.unpack("<Q", self.data[:8])[0], struct.unpack(">Q", self.data[:8])[0]
        for val, e, m in ((le8, "<", 8), (be8, ">", 8)):
            if val in (84, 164):
                self.e, self.msize, self.header_len, self.pos = e, m, val, 8
                return
        le4, be4 = struct.unpack("<I", self.data[:4])[0], struct.unpack(">I", self.data[:4])[0]
        for val, e in ((le4, "<"), (be4, ">")):
            if val in (84, 164):
                self.e, self.msize, self.header_len, self.pos = e, 4, val, 4
                return
        raise DcdError("unsupported", "unsupported DCD record marker")

    def _read_exact(self, n: int) -> bytes:
        if self.pos + n > len(self.data):
            self.pos = len(self.data)
            raise DcdError("io", "failed to fill whole buffer")
        out = self.data[self.pos:self.pos + n]
        self.pos += n
        return out

    def _marker(self) -> int:
        raw = self._read_exact(self.msize)
        return struct.unpack(self.e + ("I" if self.msize == 4 else "Q"), raw)[0]

    def _marker_opt(self) -> Optional[int]:
        if self.pos + self.msize > len(self.data):
            self.pos = len(self.data)
            return None
        return self._marker()

    def _skip_record(self, n: int, msg: str = "record length mismatch"):
        self._read_exact(n)
        if self._marker() != n:
            raise DcdError("parse", msg)

    def _axis(self, n: int) -> np.ndarray:
        if n != self.n_atoms * 4:
            raise DcdError("parse", "unexpected float record length")
        vals = np.frombuffer(self._read_exact(n), dtype=self.e + "f4").astype(np.float32)
        if self._marker() != n:
            raise DcdError("parse", "float record length mismatch")
        return vals

    def _cell(self, n: int) -> Box:
        if n == 24:
            vals = [float(x) for x in np.frombuffer(self._read_exact(24), self.e + "f4")]
        else:
            vals = [float(x) for x in np.frombuffer(self._read_exact(48), self.e + "f8")]
        if self._marker() != n:
            raise DcdError("parse", "unitcell record length mismatch")
        box = box_from_values(vals, self.charmm, float(self.scale))
        if box[0] != 0:
            return box
        return box_from_values(vals, not self.charmm, float(self.scale))

    # -- frames ----------------------------------------------------------
    def read_frame(self, selection: Optional[np.ndarray] = None, needs_box: bool = True):
        """One frame: (coords [n or n_sel][3] float32, box) or None at the end."""
        expected = self.n_atoms * 4
        n = self._marker_opt()
        if n is None:
            return None
        box = _none_box()
        if n != expected and n in (24, 48):
            if needs_box:
                box = self._cell(n)
            else:
                self._skip_record(n)
            n = self._marker_opt()
            if n is None:
                return None
        if n != expected:
            raise DcdError("parse", "unexpected DCD coordinate record length")
        x = self._axis(n)
        y = self._axis(self._marker())
        z = self._axis(self._marker())
        xyz = np.stack([x, y, z], axis=1)
        if selection is not None:
            xyz = xyz[np.asarray(selection, np.int64)]
        if self.scale != np.float32(1.0):
            xyz = (xyz * self.scale).astype(np.float32)
        return np.ascontiguousarray(xyz, np.float32), box

    def read_chunk(self, max_frames: int, selection: Optional[Sequence[int]] = None, needs_box: bool = True):
        """read_chunk / read_chunk_selected (dcd.rs:127-155): up to max_frames
        frames -> (coords [F][n][3], box kinds [F], box matrices [F][9])."""
        sel = None
        if selection is not None:
            sel = np.asarray(selection, np.int64)
            bad = sel[sel >= self.n_atoms]
            if bad.size:
                raise DcdError("mismatch", f"selection index {int(bad[0])} out of bounds for trajectory with "
                                           f"{self.n_atoms} atoms")
        frames: List[np.ndarray] = []
        kinds: List[int] = []
        mats: List[np.ndarray] = []
        while len(frames) < max_frames:
            fr = self.read_frame(sel, needs_box)
            if fr is None:
                break
            frames.append(fr[0])
            kinds.append(fr[1][0])
            mats.append(fr[1][1])
        n = self.n_atoms if sel is None else sel.size
        if not frames:
            return np.zeros((0, n, 3), np.float32), np.zeros(0, np.int32), np.zeros((0, 9), np.float32)
        return np.stack(frames), np.asarray(kinds, np.int32), np.stack(mats)

    def skip_frames(self, n: int) -> int:
        done = 0
        while done < n and self.read_frame(None, needs_box=False) is not None:
            done += 1
        return done

    def reset(self):
        self.pos = self.data_start


def read_all(path: str, length_scale: float = 1.0, selection=None, needs_box: bool = True):
    r = DcdReader(path, length_scale)
    return r.read_chunk(1 << 62, selection, needs_box)
