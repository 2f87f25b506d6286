"""Synthetic meshes in the form DMPlex + DMPlexComputeGeometryFVM hand to the FV solver.

``box_mesh`` builds the uniform quad/hex box of ``DMPlexCreateBoxMesh`` with either periodic
directions or, on non-periodic sides, one FV ghost cell behind every boundary face (what
``DMPlexConstructGhostCells`` adds; its centroid is the interior centroid reflected across the face
and its volume the interior cell's, as ``DMPlexComputeGeometryFVM`` sets them). Support order is
(interior, ghost) with the area-weighted normal pointing from the first to the second cell.

Cells are numbered x-fastest (``order="natural"``, DMPlexCreateBoxMesh's order) or along a Morton
curve (``order="morton"``: the numbering a DMPlexPermute with a space-filling-curve ordering gives,
which makes every compact block of cells contiguous in memory); faces follow their left cell. Ghost
cells follow the interior cells.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class Mesh:
    dim: int
    face_cells: np.ndarray     # (nf, 2) int32
    face_normal: np.ndarray    # (nf, 3) float64
    face_centroid: np.ndarray  # (nf, 3)
    cell_centroid: np.ndarray  # (nc, 3)
    cell_volume: np.ndarray    # (nc,)
    cell_kind: np.ndarray      # (nc,) uint8
    face_shift: np.ndarray | None = None  # (nf, 3) periodic image shift or None
    n_interior: int = 0
    shape: tuple = ()
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_cells(self) -> int:
        return int(self.cell_volume.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_cells.shape[0])

    def desc(self) -> L.MeshDesc:
        arrs = [np.ascontiguousarray(a) for a in (self.face_cells, self.face_normal, self.face_centroid,
                                                  self.cell_centroid, self.cell_volume, self.cell_kind)]
        fc, fn, fcen, cc, cv, ck = arrs
        fs = None if self.face_shift is None else np.ascontiguousarray(self.face_shift)
        self._keep = arrs + [fs]
        return L.MeshDesc(self.dim, self.n_cells, self.n_faces, L.iptr(fc), L.dptr(fn), L.dptr(fcen), L.dptr(cc),
                          L.dptr(cv), L.u8ptr(ck), L.dptr(fs) if fs is not None else None)


def _morton_keys(idx: np.ndarray, dim: int) -> np.ndarray:
    """Interleave the bits of the integer cell coordinates idx[a] (a < dim) into one key per cell."""
    key = np.zeros(idx.shape[1], dtype=np.uint64)
    for b in range(21):
        for a in range(dim):
            key |= ((idx[a].astype(np.uint64) >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + a)
    return key


def box_mesh(shape, lower=None, upper=None, periodic=None, order: str = "natural") -> Mesh:
    shape = tuple(int(n) for n in shape)
    dim = len(shape)
    if dim not in (1, 2, 3) or min(shape) < 1:
        raise ValueError("shape must have 1-3 positive entries")
    lower = np.zeros(dim) if lower is None else np.asarray(lower, float)
    upper = np.ones(dim) if upper is None else np.asarray(upper, float)
    periodic = (False,) * dim if periodic is None else tuple(bool(p) for p in periodic)
    h = (upper - lower) / np.asarray(shape)
    n_int = int(np.prod(shape))
    vol = float(np.prod(h))

    # interior cell centroids, x fastest
    idx = np.indices(shape[::-1]).reshape(dim, -1)[::-1]  # idx[a] = index along axis a, x fastest
    cc = np.zeros((n_int, 3))
    for a in range(dim):
        cc[:, a] = lower[a] + (idx[a] + 0.5) * h[a]
    strides = [int(np.prod(shape[:a])) for a in range(dim)]

    fcs, fns, fcents, fshifts = [], [], [], []
    ghost_cent, ghost_of = [], []
    n_ghost = 0
    for a in range(dim):
        area = float(np.prod([h[b] for b in range(dim) if b != a])) if dim > 1 else 1.0
        ia = idx[a]
        cells = np.arange(n_int)
        # interior faces: cell with index i along a and its +a neighbour
        lo = cells[ia < shape[a] - 1]
        if lo.size:
            hi = lo + strides[a]
            fc = np.stack([lo, hi], 1)
            fcen = cc[lo].copy()
            fcen[:, a] += 0.5 * h[a]
            fcs.append(fc)
            fcents.append(fcen)
            n = np.zeros((lo.size, 3))
            n[:, a] = area
            fns.append(n)
            fshifts.append(np.zeros((lo.size, 3)))
        last = cells[ia == shape[a] - 1]
        first = last - (shape[a] - 1) * strides[a]
        if periodic[a]:
            fc = np.stack([last, first], 1)
            fcen = cc[last].copy()
            fcen[:, a] += 0.5 * h[a]
            n = np.zeros((last.size, 3))
            n[:, a] = area
            sh = np.zeros((last.size, 3))
            sh[:, a] = upper[a] - lower[a]
            fcs.append(fc)
            fcents.append(fcen)
            fns.append(n)
            fshifts.append(sh)
        else:
            for side, cl in ((-1, first), (+1, last)):
                g = n_int + n_ghost + np.arange(cl.size)
                n_ghost += cl.size
                fc = np.stack([cl, g], 1)
                fcen = cc[cl].copy()
                fcen[:, a] += side * 0.5 * h[a]
                n = np.zeros((cl.size, 3))
                n[:, a] = side * area
                gcen = 2.0 * fcen - cc[cl]
                fcs.append(fc)
                fcents.append(fcen)
                fns.append(n)
                fshifts.append(np.zeros((cl.size, 3)))
                ghost_cent.append(gcen)
                ghost_of.append(cl)
    face_cells = np.concatenate(fcs).astype(np.int32)
    face_normal = np.concatenate(fns)
    face_centroid = np.concatenate(fcents)
    face_shift = np.concatenate(fshifts)
    if order == "morton":
        # renumber interior cells along the Morton curve, then sort faces by their left cell
        key = _morton_keys(idx, dim)
        perm = np.argsort(key, kind="stable")          # new -> old
        rank = np.empty(n_int, np.int64)
        rank[perm] = np.arange(n_int)                   # old -> new
        cc = cc[perm]
        fc = face_cells.astype(np.int64)
        interior = fc < n_int
        fc[interior] = rank[fc[interior]]
        fo = np.lexsort((fc[:, 1], fc[:, 0]))
        face_cells = fc[fo].astype(np.int32)
        face_normal = face_normal[fo]
        face_centroid = face_centroid[fo]
        face_shift = face_shift[fo]
        # ghost cells keep their creation order; their interior partners were renumbered above
    elif order != "natural":
        raise ValueError("order must be 'natural' or 'morton'")
    if n_ghost:
        cc = np.concatenate([cc] + ghost_cent)
    nc = n_int + n_ghost
    cell_volume = np.full(nc, vol)
    kind = np.zeros(nc, np.uint8)
    kind[n_int:] = L.CELL_BOUNDARY
    any_periodic = any(periodic)
    return Mesh(dim=dim, face_cells=face_cells, face_normal=face_normal, face_centroid=face_centroid,
                cell_centroid=cc, cell_volume=cell_volume, cell_kind=kind,
                face_shift=face_shift if any_periodic else None, n_interior=n_int, shape=shape)


def ghost_interior_map(mesh: Mesh) -> np.ndarray:
    """For every boundary ghost cell (in order), the interior cell across its face."""
    g = np.nonzero(mesh.cell_kind == L.CELL_BOUNDARY)[0]
    out = np.empty(g.size, np.int64)
    fc = mesh.face_cells
    is_g = mesh.cell_kind[fc[:, 1]] == L.CELL_BOUNDARY
    out_map = dict(zip(fc[is_g, 1].tolist(), fc[is_g, 0].tolist()))
    for i, c in enumerate(g.tolist()):
        out[i] = out_map[c]
    return out
