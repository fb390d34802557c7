"""Lattices in MARQOV's form, lowered to engine lattice descriptors.

* ``RegularHypercubic(len, dim)`` / ``FixedDimRegularHypercubic(dim, len)``:
  periodic hypercubic lattices (src/lattice/regular_hypercubic.h:15-143); the
  engine runs them on its stencil path (checkerboard colours, even ``len``).
* ``CSRLattice``: any lattice given by its neighbour lists in ``nbrs(0, i)``
  order (the reference lattice concept), with optional symmetric bonds
  (``bnds``) and an optional proper colouring (else the engine colours
  greedily).  ``from_nbrs`` lowers any object with ``size()`` / ``nbrs()`` /
  optional ``bnds()``, the way a reference lattice plugs in.
* ``BondedHypercubic``: a hypercubic lattice with bond weights, kept on the
  stencil path.
* Builders for the synthetic workloads: ``RegularRandomBond`` (bimodal +-1
  bonds on a hypercubic lattice, src/lattice/regular_random_bond.h:13-77 with a
  seeded generator) and ``RandomGeometricGraph2D`` (periodic unit square).
"""
from __future__ import annotations

import re

import numpy as np

from . import _lib as L


class Lattice:
    def desc(self) -> L.LatticeDesc:  # pragma: no cover - abstract
        raise NotImplementedError

    def size(self) -> int:  # pragma: no cover - abstract
        raise NotImplementedError


class RegularHypercubic(Lattice):
    def __init__(self, len: int, dim: int):  # noqa: A002 - reference argument name
        self.len = int(len)
        self.dim = int(dim)
        self.npoints = self.len ** self.dim

    def size(self) -> int:
        return self.npoints

    def nbrs(self, alpha: int, i: int) -> list[int]:
        """Neighbours in the reference order +x,-x,+y,-y,... (regular_hypercubic.h:31-66)."""
        out = []
        p = 1
        for _ in range(self.dim):
            pl = p * self.len
            base = (i // pl) * pl
            out.append(base + (i + p) % pl)
            c = i - p
            out.append(base + (c + pl) % pl if c < base else c)
            p = pl
        return out

    def crds(self, k: int) -> list[float]:
        """Site coordinates (x + 0.5) / len (regular_hypercubic.h:73-85)."""
        a = 1.0 / self.len
        out = []
        p = 1
        for _ in range(self.dim):
            out.append(((k // p) % self.len) * a + 0.5 * a)
            p *= self.len
        return out

    def desc(self) -> L.LatticeDesc:
        return L.LatticeDesc(kind=L.LATTICE_HYPERCUBIC, dim=self.dim, len=self.len)

    def to_csr(self) -> "CSRLattice":
        n, d = self.npoints, self.dim
        idx = np.arange(n, dtype=np.int64)
        cols = np.empty((n, 2 * d), np.int32)
        p = 1
        for j in range(d):
            pl = p * self.len
            base = (idx // pl) * pl
            cols[:, 2 * j] = base + (idx + p) % pl
            c = idx - p
            cols[:, 2 * j + 1] = np.where(c < base, base + (c + pl) % pl, c)
            p = pl
        rp = np.arange(0, n * 2 * d + 1, 2 * d, dtype=np.int32)
        par = np.zeros(n, np.int64)
        p = 1
        for j in range(d):
            par += (idx // p) % self.len
            p *= self.len
        return CSRLattice(rp, cols.reshape(-1), colours=(par & 1).astype(np.int32))


class SimpleBipartite(RegularHypercubic):
    """``SimpleBipartite(len, dim)`` (src/lattice/simple_bipartite.h:8-58): the
    periodic hypercubic lattice with a ``termselector`` -- a site whose
    coordinate sum is even (sublattice A) takes onsite term 0 only, an odd one
    term 1 only (``identify``, simple_bipartite.h:22-36).  Runs on the stencil
    path; the sublattice of a site is its checkerboard colour."""

    def __init__(self, len: int, dim: int):  # noqa: A002 - reference argument name
        if int(len) % 2:
            raise ValueError("SimpleBipartite needs an even linear size")
        super().__init__(len, dim)

    def identify(self, k: int) -> int:
        s = 0
        for _ in range(self.dim):
            s += k % self.len
            k //= self.len
        return s % 2

    def termselector(self, rsite: int) -> list[int]:
        return [self.identify(rsite)]

    def desc(self) -> L.LatticeDesc:
        return L.LatticeDesc(kind=L.LATTICE_BIPARTITE, dim=self.dim, len=self.len)


def FixedDimRegularHypercubic(dim: int, len: int) -> RegularHypercubic:  # noqa: A002
    """``FixedDimRegularHypercubic<dim>(len)``."""
    return RegularHypercubic(len, dim)


class CSRLattice(Lattice):
    def __init__(self, row_ptr, col_idx, bonds=None, colours=None, crds=None):
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.bonds = None if bonds is None else np.ascontiguousarray(bonds, np.int8)
        self.colours = None if colours is None else np.ascontiguousarray(colours, np.int32)
        self.coords = crds
        self.n = len(self.row_ptr) - 1

    @classmethod
    def from_nbrs(cls, lat, with_bonds: bool | None = None, colours=None) -> "CSRLattice":
        """Lower any reference-style lattice (``size()``, ``nbrs(0, i)``, optional
        ``bnds(0, i)``) by querying it once per site."""
        n = int(lat.size())
        rp = np.zeros(n + 1, np.int32)
        cols, bnds = [], []
        has_b = hasattr(lat, "bnds") if with_bonds is None else with_bonds
        for i in range(n):
            nb = list(lat.nbrs(0, i))
            cols.extend(nb)
            if has_b:
                bnds.extend(list(lat.bnds(0, i)))
            rp[i + 1] = rp[i] + len(nb)
        return cls(rp, np.array(cols, np.int32), np.array(bnds, np.int8) if has_b else None, colours)

    def size(self) -> int:
        return self.n

    def nbrs(self, alpha: int, i: int):
        return self.col_idx[self.row_ptr[i]:self.row_ptr[i + 1]].tolist()

    def crds(self, i: int) -> list[float]:
        """Site coordinates as given (none for a lattice built without)."""
        return [] if self.coords is None else [float(c) for c in self.coords[i]]

    def bnds(self, alpha: int, i: int):
        if self.bonds is None:
            raise AttributeError("lattice has no bonds")
        return self.bonds[self.row_ptr[i]:self.row_ptr[i + 1]].tolist()

    def desc(self) -> L.LatticeDesc:
        return L.LatticeDesc(kind=L.LATTICE_CSR, n=self.n, row_ptr=self.row_ptr.ctypes.data,
                             col_idx=self.col_idx.ctypes.data,
                             bonds=None if self.bonds is None else self.bonds.ctypes.data,
                             colours=None if self.colours is None else self.colours.ctypes.data)

    def greedy_colours(self) -> np.ndarray:
        """Greedy colouring in site order (the engine's default)."""
        col = np.full(self.n, -1, np.int32)
        for i in range(self.n):
            used = {int(col[j]) for j in self.col_idx[self.row_ptr[i]:self.row_ptr[i + 1]] if col[j] >= 0}
            c = 0
            while c in used:
                c += 1
            col[i] = c
        return col


class BondedHypercubic(RegularHypercubic):
    """A periodic hypercubic lattice with symmetric bond weights ``bnds``,
    given per site in the ``nbrs(0, i)`` order +x,-x,+y,-y,... (an n x 2 dim
    int8 array).  The engine keeps it on the stencil path and stores one plane
    of +d bonds per dimension; ``to_csr()`` gives the same lattice as CSR."""

    def __init__(self, len: int, dim: int, bonds):  # noqa: A002 - reference argument name
        super().__init__(len, dim)
        self.bonds = np.ascontiguousarray(bonds, np.int8).reshape(self.npoints, 2 * self.dim)

    def bnds(self, alpha: int, i: int):
        return self.bonds[i].tolist()

    def desc(self) -> L.LatticeDesc:
        return L.LatticeDesc(kind=L.LATTICE_HYPERCUBIC, dim=self.dim, len=self.len, bonds=self.bonds.ctypes.data)

    def to_csr(self) -> "CSRLattice":
        base = super().to_csr()
        return CSRLattice(base.row_ptr, base.col_idx, self.bonds.reshape(-1), base.colours)


def RegularRandomBond(len: int, dim: int, p: float = 0.5, seed: int = 0) -> BondedHypercubic:  # noqa: A002
    """Hypercubic lattice with symmetric bimodal +-1 bonds, P(+1) = p: the
    ``RegularRandomBond<BimodalPDF>`` lattice (regular_random_bond.h:26-55) with
    a seeded generator instead of ``random_device``.  Each undirected bond gets
    one draw; both of its entries carry it."""
    base = RegularHypercubic(len, dim).to_csr()
    n = base.n
    rng = np.random.default_rng(seed)
    deg = 2 * dim
    cols = base.col_idx.reshape(n, deg)
    w = np.where(rng.random((n, dim)) < p, 1, -1).astype(np.int8)  # forward bond of each dim
    bonds = np.empty((n, deg), np.int8)
    for j in range(dim):
        bonds[:, 2 * j] = w[:, j]                        # +dir bond owned by the site
        bonds[:, 2 * j + 1] = w[cols[:, 2 * j + 1], j]   # -dir bond owned by the neighbour
    return BondedHypercubic(len, dim, bonds)


def RandomGeometricGraph2D(n: int, mean_degree: float = 8.0, seed: int = 0) -> CSRLattice:
    """n points uniform in the periodic unit square, bonds between points closer
    than r with pi r^2 n = mean_degree.  Neighbour lists sorted by id; cell-list
    construction, O(n)."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    r = float(np.sqrt(mean_degree / (np.pi * n)))
    nc = max(1, int(1.0 / r))
    cell = np.minimum((pts * nc).astype(np.int64), nc - 1)
    cid = cell[:, 0] * nc + cell[:, 1]
    order = np.argsort(cid, kind="stable")
    starts = np.searchsorted(cid[order], np.arange(nc * nc + 1))
    src, dst = [], []
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            ncell = ((cell[:, 0] + dx) % nc) * nc + (cell[:, 1] + dy) % nc
            cnt = starts[ncell + 1] - starts[ncell]
            tot = int(cnt.sum())
            if tot == 0:
                continue
            a = np.repeat(np.arange(n), cnt)
            off = np.arange(tot) - np.repeat(np.cumsum(cnt) - cnt, cnt)
            b = order[np.repeat(starts[ncell], cnt) + off]
            d = pts[a] - pts[b]
            d -= np.round(d)
            keep = (a != b) & ((d * d).sum(1) < r * r)
            src.append(a[keep])
            dst.append(b[keep])
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    if nc < 3:  # small grids visit a cell more than once
        pair = np.unique(np.stack([src, dst], 1), axis=0)
        src, dst = pair[:, 0], pair[:, 1]
    o = np.lexsort((dst, src))
    src, dst = src[o], dst[o]
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, src + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    return CSRLattice(rp, dst.astype(np.int32), crds=pts)


_STOI = re.compile(r"\s*([+-]?\d+)")
_STOD = re.compile(r"\s*([+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan))", re.IGNORECASE)


def _stoi(field: str) -> int:
    """std::stoi: leading blanks, sign and digits; the rest is ignored."""
    m = _STOI.match(field)
    if not m:
        raise ValueError(f"not an integer: {field!r}")
    return int(m.group(1))


def _stod(field: str) -> float:
    """std::stod on a decimal field: the longest leading number."""
    m = _STOD.match(field)
    if not m:
        raise ValueError(f"not a number: {field!r}")
    return float(m.group(1))


def read_graph_csv(path: str, idxoffs: int = 0) -> CSRLattice:
    """GraphFromCSV(filename) (src/lattice/graph_from_csv.h:40-44) over
    import_geometry_ncoords / import_geometry (src/lattice/util/io.h:60-126):
    line 1 holds the number of coordinates c (std::stoi), line 2 is a header
    and is skipped, every further line is one site: tab-separated fields, the
    first c coordinates (std::stod), the rest neighbour ids (std::stoi, minus
    idxoffs).  An empty line is a site without coordinates or neighbours,
    except the empty remainder after the last newline; an empty field
    between two tabs is an error, as std::stod / std::stoi of "" is there."""
    with open(path, newline="") as fh:
        rows = fh.read().split("\n")
    ncoords = _stoi(rows[0])
    body = rows[2:]
    if body and body[-1] == "":
        body = body[:-1]
    rp, cols, crd = [0], [], []
    for row in body:
        fields = row.split("\t") if row else []
        if fields and fields[-1] == "":
            fields = fields[:-1]  # a trailing tab ends the line, it opens no field
        crd.append([_stod(x) for x in fields[:ncoords]])
        nb = [_stoi(x) - idxoffs for x in fields[ncoords:]]
        cols.extend(nb)
        rp.append(rp[-1] + len(nb))
    rect = all(len(c) == len(crd[0]) for c in crd) if crd else True
    return CSRLattice(np.array(rp, np.int32), np.array(cols, np.int32),
                      crds=np.array(crd, np.float64) if rect else crd)


def save_geometry(lattice, path: str) -> None:
    """save_geometry(grid, path) (src/lattice/util/io.h:34-52): one line per
    site, the count of neighbours plus coordinates, then tab-separated the
    coordinates (fixed, 16 decimals) and the neighbour ids.  As in the
    reference, the file has no header lines, so read_graph_csv does not read
    it back."""
    with open(path, "w", newline="") as fh:
        for i in range(int(lattice.size())):
            nb = list(lattice.nbrs(0, i))
            cr = list(lattice.crds(i))
            fh.write(str(len(nb) + len(cr)) + "".join("\t%.16f" % float(c) for c in cr)
                     + "".join("\t%d" % int(j) for j in nb) + "\n")
