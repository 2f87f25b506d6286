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


def delaunay_mesh(n_cells: int, extent=(1.0, 0.2, 0.2), seed: int = 20261205, jitter: float = 0.3) -> Mesh:
    """Tetrahedral mesh of the box [0, extent] from the Delaunay triangulation of a seeded point cloud
    (a lattice of spacing h jittered by up to jitter*h, with the box corners and the lattice points on
    the box faces held on the faces, so the tetrahedra fill the box), with one FV ghost cell behind
    every boundary face (centroid reflected through the face centroid, the interior volume).
    n_cells sets the lattice spacing; the tetrahedron count comes out near it. Cells are ordered along
    a Morton curve of their centroids."""
    from scipy.spatial import Delaunay

    ext = np.asarray(extent, float)
    # about 6.6 tetrahedra per lattice point for a jittered lattice
    h = (float(np.prod(ext)) * 6.6 / n_cells) ** (1.0 / 3.0)
    shape = np.maximum(1, np.round(ext / h).astype(int))
    axes = [np.linspace(0.0, ext[a], shape[a] + 1) for a in range(3)]
    P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    hs = ext / shape
    J = rng.uniform(-jitter, jitter, P.shape) * hs
    on_face = (np.isclose(P, 0.0) | np.isclose(P, ext))  # keep boundary points on their faces
    J[on_face] = 0.0
    P = P + J
    # joggled input (QJ): Qhull perturbs the lattice's cospherical points instead of resolving them,
    # five times faster here; the tetrahedra refer to the unperturbed points
    tri = Delaunay(P, qhull_options="Qbb Qc Q12 QJ")
    tets = tri.simplices.astype(np.int64)
    V = P[tets]  # (nt, 4, 3)
    vol6 = np.einsum("ij,ij->i", V[:, 1] - V[:, 0], np.cross(V[:, 2] - V[:, 0], V[:, 3] - V[:, 0]))
    keep = np.abs(vol6) > 1e-12 * float(np.prod(hs))  # drop flat boundary slivers
    tets, V, vol6 = tets[keep], V[keep], vol6[keep]
    cc = V.mean(1)
    # Morton order of the cells
    q = ((cc / ext) * ((1 << 20) - 1)).astype(np.int64).T
    perm = np.argsort(_morton_keys(q, 3), kind="stable")
    tets, V, vol6, cc = tets[perm], V[perm], vol6[perm], cc[perm]
    nt = tets.shape[0]
    # faces: the 4 vertex triples of every tet, matched by their sorted vertex ids
    tri_idx = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
    F = np.sort(tets[:, tri_idx].reshape(-1, 3), axis=1)
    owner = np.repeat(np.arange(nt), 4)
    key = (F[:, 0] * P.shape[0] + F[:, 1]) * P.shape[0] + F[:, 2]
    order = np.argsort(key, kind="stable")
    ks, os_ = key[order], owner[order]
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    inner = np.zeros(ks.size, bool)
    inner[same] = inner[same + 1] = True
    pairs = np.stack([os_[same], os_[same + 1]], 1)
    bnd_pos = order[~inner]
    bnd_cells = owner[bnd_pos]
    tri_int = F[order[same]]
    tri_bnd = F[bnd_pos]
    # interior faces (left = smaller cell id), then boundary faces with their ghosts
    L_, R_ = pairs.min(1), pairs.max(1)
    nb = bnd_cells.size
    ghosts = nt + np.arange(nb)
    face_cells = np.concatenate([np.stack([L_, R_], 1), np.stack([bnd_cells, ghosts], 1)])
    tris = np.concatenate([tri_int, tri_bnd])
    Pt = P[tris]
    fcen = Pt.mean(1)
    nrm = 0.5 * np.cross(Pt[:, 1] - Pt[:, 0], Pt[:, 2] - Pt[:, 0])
    gcen = 2.0 * fcen[L_.size:] - cc[bnd_cells]
    cell_centroid = np.concatenate([cc, gcen])
    # orient every normal from left to right
    d = cell_centroid[face_cells[:, 1]] - cell_centroid[face_cells[:, 0]]
    nrm[np.einsum("ij,ij->i", nrm, d) < 0] *= -1.0
    fo = np.lexsort((face_cells[:, 1], face_cells[:, 0]))
    cell_volume = np.concatenate([np.abs(vol6) / 6.0, np.abs(vol6[bnd_cells]) / 6.0])
    kind = np.zeros(nt + nb, np.uint8)
    kind[nt:] = L.CELL_BOUNDARY
    return Mesh(dim=3, face_cells=face_cells[fo].astype(np.int32), face_normal=nrm[fo], face_centroid=fcen[fo],
                cell_centroid=cell_centroid, cell_volume=cell_volume, cell_kind=kind, face_shift=None, n_interior=nt, shape=())
