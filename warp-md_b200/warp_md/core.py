"""System / Selection / Trajectory: the in-memory inputs of the RMSD plans.

Shapes and behaviour follow the reference bindings:
  * ``System.from_arrays(atom_table, positions0=None)`` (crates/traj-py/src/io.rs:104+):
    atom_table is a mapping or object with a ``name`` sequence and optional
    ``resname``, ``resid``, ``mass``, ``element``, ``chain``/``chain_id``;
  * ``system.select(expr)`` (io.rs:255-259) over the selection grammar of
    crates/traj-core/src/selection_expression.rs (all, name, resname, resid
    with ``a-b`` / ``a:b`` ranges, chain, element, and/or/not, parentheses);
    ``select_indices`` (io.rs:261-267) takes explicit indices;
  * ``Trajectory.from_numpy(coords, box=None, time_ps=None)`` (io.rs:670-685):
    coords (frames, atoms, 3) or (atoms, 3), float32 or float64 (stored as
    float32, as the reference converts to [f32; 4]).
"""
from __future__ import annotations

from typing import Any, List, Optional, Sequence

import numpy as np


def _field(table: Any, key: str):
    if isinstance(table, dict):
        return table.get(key)
    if hasattr(table, key):
        return getattr(table, key)
    try:
        return table[key]
    except (KeyError, TypeError, IndexError):
        return None


class Selection:
    """Atom indices picked by a selection expression (PySelection)."""

    def __init__(self, indices: Sequence[int], expr: str = "__indices__"):
        self._indices = np.asarray(indices, dtype=np.uint32).copy()
        self.expr = expr

    @property
    def indices(self) -> List[int]:
        return self._indices.tolist()

    def as_array(self) -> np.ndarray:
        return self._indices

    def __len__(self) -> int:
        return int(self._indices.shape[0])


class System:
    """Topology (atom table) plus optional reference coordinates positions0."""

    def __init__(self, names, resnames, resids, masses, elements, chains, positions0):
        self.names = [str(n).strip().upper() for n in names]
        n = len(self.names)
        self.resnames = [str(r).strip().upper() for r in resnames] if resnames is not None else [""] * n
        self.resids = np.asarray(resids if resids is not None else np.zeros(n), dtype=np.int64)
        self.masses = np.asarray(masses if masses is not None else np.ones(n), dtype=np.float32)
        self.elements = [str(e).strip().upper() for e in elements] if elements is not None else [""] * n
        self.chains = [str(c).strip().upper() for c in chains] if chains is not None else [""] * n
        for arr, label in ((self.resnames, "resname"), (self.resids, "resid"), (self.masses, "mass"),
                           (self.elements, "element"), (self.chains, "chain")):
            if len(arr) != n:
                raise RuntimeError("atom_table fields must all have the same length")
        self.positions0 = None
        if positions0 is not None:
            p = np.asarray(positions0, dtype=np.float32)
            if p.ndim != 2 or p.shape[1] != 3 or p.shape[0] != n:
                raise RuntimeError("positions0 must have shape (n_atoms, 3)")
            self.positions0 = np.ascontiguousarray(p)

    @staticmethod
    def from_arrays(atom_table: Any, positions0: Optional[Any] = None) -> "System":
        names = _field(atom_table, "name")
        if names is None:
            raise RuntimeError("atom_table requires 'name'")
        chains = _field(atom_table, "chain")
        if chains is None:
            chains = _field(atom_table, "chain_id")
        return System(list(names), _field(atom_table, "resname"), _field(atom_table, "resid"),
                      _field(atom_table, "mass"), _field(atom_table, "element"), chains, positions0)

    def n_atoms(self) -> int:
        return len(self.names)

    def atom_table(self) -> dict:
        return {"name": list(self.names), "resname": list(self.resnames), "resid": self.resids.tolist(),
                "mass": self.masses.tolist(), "element": list(self.elements), "chain": list(self.chains)}

    def select(self, expr: str) -> Selection:
        mask = _SelectionParser(expr, self).parse()
        return Selection(np.nonzero(mask)[0], expr)

    def select_indices(self, indices: Sequence[int]) -> Selection:
        return Selection(indices)


class Trajectory:
    """In-memory trajectory (MemoryTraj, io.rs:612-659), float32 (frames, atoms, 3)."""

    def __init__(self, coords: np.ndarray, box=None, time_ps=None):
        self.coords = coords
        self.box = box
        self.time_ps = time_ps

    @staticmethod
    def from_numpy(coords: Any, box: Optional[Any] = None, time_ps: Optional[Any] = None) -> "Trajectory":
        a = np.asarray(coords)
        if a.dtype not in (np.float32, np.float64):
            raise RuntimeError("coords must be a numpy array with shape (frames, atoms, 3) or (atoms, 3)")
        if a.ndim == 2:
            a = a[None]
        if a.ndim != 3:
            raise RuntimeError("coords must have shape (frames, atoms, 3) or (atoms, 3)")
        if a.shape[2] != 3:
            raise RuntimeError("coords must have final dimension 3")
        return Trajectory(np.ascontiguousarray(a, dtype=np.float32), box, time_ps)

    @staticmethod
    def open_dcd(path: str, system: "System", length_scale: Optional[float] = None) -> "Trajectory":
        """A DCD file (PyTrajectory.open_dcd, crates/traj-py/src/io.rs:687-708)
        read through the GPU decoder; see warp_md.dcd."""
        from .dcd import DcdTrajectory

        return DcdTrajectory(path, system, length_scale)

    @staticmethod
    def open_xtc(path: str, system: "System") -> "Trajectory":
        """XTC needs the xdrfile codec, which this build does not provide."""
        raise RuntimeError("unsupported: XTC trajectories are not provided by this build (use DCD or from_numpy)")

    def n_atoms(self) -> int:
        return int(self.coords.shape[1])

    def n_frames(self) -> int:
        return int(self.coords.shape[0])

    def count_frames(self, chunk_frames: Optional[int] = None) -> int:
        return self.n_frames()


# ---------------------------------------------------------------------------
# selection grammar: or > and > not > primary
# ---------------------------------------------------------------------------

_KEYWORDS = {"and", "or", "not", "all", "name", "resname", "resid", "chain", "element", "protein", "backbone",
             "sidechain"}


def _tokenize(expr: str) -> List[str]:
    out: List[str] = []
    cur = ""
    for ch in expr:
        if ch.isspace() or ch in "():":
            if cur:
                out.append(cur)
                cur = ""
            if ch in "():":
                out.append(ch)
        else:
            cur += ch
    if cur:
        out.append(cur)
    return out


def _is_boundary(tok: str) -> bool:
    return tok in ("(", ")", ":") or tok.lower() in _KEYWORDS


class _SelectionParser:
    def __init__(self, expr: str, system: System):
        self.toks = _tokenize(expr)
        self.pos = 0
        self.sys = system
        self.n = system.n_atoms()

    def _peek(self) -> Optional[str]:
        return self.toks[self.pos] if self.pos < len(self.toks) else None

    def _next(self) -> Optional[str]:
        t = self._peek()
        if t is not None:
            self.pos += 1
        return t

    def parse(self) -> np.ndarray:
        if not self.toks:
            return np.ones(self.n, bool)
        m = self._or()
        if self._peek() is not None:
            raise RuntimeError(f"invalid selection: unexpected token '{self._peek()}'")
        return m

    def _or(self):
        m = self._and()
        while (self._peek() or "").lower() == "or":
            self._next()
            m = m | self._and()
        return m

    def _and(self):
        m = self._not()
        while (self._peek() or "").lower() == "and":
            self._next()
            m = m & self._not()
        return m

    def _not(self):
        if (self._peek() or "").lower() == "not":
            self._next()
            return ~self._not()
        return self._primary()

    def _values(self) -> List[str]:
        vals = []
        while self._peek() is not None and not _is_boundary(self._peek()):
            vals.append(self._next().upper())
        if not vals:
            raise RuntimeError("invalid selection: expected value after keyword")
        return vals

    def _resids(self):
        ranges = []
        while self._peek() is not None and not _is_boundary(self._peek()):
            tok = self._next()
            split = next((i for i, c in enumerate(tok) if i > 0 and c in "-:"), None)
            if split is not None:
                ranges.append((self._int(tok[:split]), self._int(tok[split + 1:])))
                continue
            start = self._int(tok)
            if self._peek() == ":":
                self._next()
                end_tok = self._next()
                if end_tok is None or _is_boundary(end_tok):
                    raise RuntimeError("invalid selection: expected resid after ':'")
                ranges.append((start, self._int(end_tok)))
            else:
                ranges.append((start, start))
        if not ranges:
            raise RuntimeError("invalid selection: expected resid value")
        return ranges

    @staticmethod
    def _int(tok: str) -> int:
        try:
            return int(tok)
        except ValueError:
            raise RuntimeError(f"invalid selection: invalid residue id '{tok}'") from None

    def _primary(self):
        tok = self._peek()
        if tok is None:
            raise RuntimeError("invalid selection: unexpected end of selection")
        if tok == "(":
            self._next()
            m = self._or()
            if self._next() != ")":
                raise RuntimeError("invalid selection: expected ')'")
            return m
        kw = tok.lower()
        s = self.sys
        if kw == "all":
            self._next()
            return np.ones(self.n, bool)
        if kw in ("name", "resname", "chain", "element"):
            self._next()
            vals = set(self._values())
            col = {"name": s.names, "resname": s.resnames, "chain": s.chains, "element": s.elements}[kw]
            return np.array([v in vals for v in col], bool)
        if kw == "resid":
            self._next()
            m = np.zeros(self.n, bool)
            for a, b in self._resids():
                m |= (s.resids >= a) & (s.resids <= b)
            return m
        if kw in ("protein", "backbone", "sidechain"):
            raise RuntimeError(f"invalid selection: '{kw}' is not provided by this build")
        raise RuntimeError(f"invalid selection: unexpected token '{tok}'")
