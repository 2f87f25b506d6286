"""Partitioned RHS over several GPUs: cell partition, two-layer halo, and the halo exchange.

Owner-computes over a cell partition, as ABLATE runs under MPI (a DMPlex distributed with a ghost
overlap, src/domain/modifiers/distributeWithGhostCells.cpp:10-14). Every rank holds

* its owned cells (kind OWNED), whose residual rows it computes;
* HALO cells: the other ranks' cells adjacent to an owned cell. The rank recomputes their limited
  least-squares gradients locally instead of exchanging gradients (the reference exchanges them,
  src/finiteVolume/cellInterpolant.cpp:490-491);
* HALO_OUTER cells: the cells adjacent to a HALO cell, whose values those gradients read;
* the boundary ghost cells adjacent to owned or HALO cells (kind BOUNDARY). A ghost belongs to the
  rank that owns its interior neighbour.

Before every RHS the rows of the cells a rank does not own are refreshed from their owners (the
DMGlobalToLocal broadcast, src/solver/timeStepper.cpp:343-344). Faces on a partition boundary are
computed by both owners, each for its own cells, so the residual needs no reduction (the
LocalToGlobal ADD at src/solver/timeStepper.cpp:379-380 has nothing to add). A local mesh keeps the
global order of its faces, so every owned cell sees its faces in the same order as in the
undistributed mesh, and the partitioned residual equals the single-domain one bit for bit.

The exchange packs the owned rows each neighbour needs with abl_rows_gather, moves them with NCCL
point-to-point (torch.distributed.batch_isend_irecv on the current stream), and unpacks them with
abl_rows_scatter.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .mesh import Mesh, _morton_keys, box_mesh


@dataclass
class LocalDomain:
    """One rank's local mesh and, per local cell, its global id and owning rank."""
    mesh: Mesh
    gid: np.ndarray    # (n_local,) int64
    owner: np.ndarray  # (n_local,) int32
    rank: int
    nparts: int

    @property
    def owned(self) -> np.ndarray:
        return self.mesh.cell_kind == L.CELL_OWNED

    def needs(self) -> dict:
        """Global ids this rank receives, per owning rank, ascending: every local cell it does not own."""
        other = self.owner != self.rank
        out = {}
        for p in np.unique(self.owner[other]):
            out[int(p)] = np.sort(self.gid[other & (self.owner == p)])
        return out


def partition_cells(mesh: Mesh, nparts: int) -> np.ndarray:
    """Part of every cell: the interior cells sorted along a Morton curve of their centroids and cut into
    nparts runs of (nearly) equal length; each boundary ghost goes with its interior neighbour."""
    kind = mesh.cell_kind
    interior = np.nonzero(kind != L.CELL_BOUNDARY)[0]
    x = mesh.cell_centroid[interior, :mesh.dim]
    lo, hi = x.min(0), x.max(0)
    span = np.where(hi > lo, hi - lo, 1.0)
    q = ((x - lo) / span * ((1 << 20) - 1)).astype(np.int64).T
    order = interior[np.argsort(_morton_keys(q, mesh.dim), kind="stable")]
    part = np.full(mesh.n_cells, -1, np.int32)
    bounds = np.linspace(0, order.size, nparts + 1).round().astype(np.int64)
    for p in range(nparts):
        part[order[bounds[p]:bounds[p + 1]]] = p
    fc = mesh.face_cells
    for a, b in ((0, 1), (1, 0)):
        g = kind[fc[:, b]] == L.CELL_BOUNDARY
        part[fc[g, b]] = part[fc[g, a]]
    return part


def submesh(mesh: Mesh, part: np.ndarray, rank: int) -> LocalDomain:
    """The local mesh of `rank`: owned cells, the two-layer halo and the ghosts they touch."""
    kind = mesh.cell_kind
    fc = mesh.face_cells.astype(np.int64)
    n = mesh.n_cells
    interior = kind != L.CELL_BOUNDARY
    owned = interior & (part == rank)

    def neighbours(mask):
        hit = np.zeros(n, bool)
        a, b = fc[:, 0], fc[:, 1]
        hit[b[mask[a]]] = True
        hit[a[mask[b]]] = True
        return hit

    halo = neighbours(owned) & interior & ~owned
    outer = neighbours(halo) & interior & ~owned & ~halo
    ghosts = neighbours(owned | halo) & ~interior
    cells = np.concatenate([np.nonzero(owned)[0], np.nonzero(halo)[0], np.nonzero(outer)[0], np.nonzero(ghosts)[0]])
    lkind = np.concatenate([np.full(owned.sum(), L.CELL_OWNED), np.full(halo.sum(), L.CELL_HALO),
                            np.full(outer.sum(), L.CELL_HALO_OUTER), np.full(ghosts.sum(), L.CELL_BOUNDARY)]).astype(np.uint8)
    local = np.full(n, -1, np.int64)
    local[cells] = np.arange(cells.size)
    core = owned | halo
    keep = (local[fc[:, 0]] >= 0) & (local[fc[:, 1]] >= 0) & (core[fc[:, 0]] | core[fc[:, 1]])
    faces = np.nonzero(keep)[0]  # global face order
    m = Mesh(mesh.dim, local[fc[faces]].astype(np.int32), mesh.face_normal[faces].copy(), mesh.face_centroid[faces].copy(),
             mesh.cell_centroid[cells].copy(), mesh.cell_volume[cells].copy(), lkind,
             None if mesh.face_shift is None else mesh.face_shift[faces].copy(), n_interior=int(owned.sum()))
    return LocalDomain(m, cells.astype(np.int64), part[cells].astype(np.int32), rank, int(part.max()) + 1)


def slab_domain(shape, nparts: int, rank: int, halo: int = 2, order: str = "morton") -> LocalDomain:
    """One rank's slab of the periodic unit box `shape`, cut along x into nparts equal slabs, built
    directly (the global mesh is never formed). Global ids are x-fastest natural box numbers."""
    nxg, ny, nz = (int(v) for v in shape)
    if nxg % nparts:
        raise ValueError("the x extent must divide into the parts")
    nx = nxg // nparts
    if nparts == 1:
        m = box_mesh(shape, periodic=(True, True, True), order=order)
        ijk = np.floor(m.cell_centroid * np.array(shape)).astype(np.int64)
        gid = ijk[:, 0] + nxg * (ijk[:, 1] + ny * ijk[:, 2])
        return LocalDomain(m, gid, np.zeros(m.n_cells, np.int32), 0, 1)
    if nx < halo:
        raise ValueError("slabs thinner than the halo")
    hx = 1.0 / nxg
    lo = (rank * nx - halo) * hx
    m = box_mesh((nx + 2 * halo, ny, nz), lower=(lo, 0.0, 0.0), upper=(lo + (nx + 2 * halo) * hx, 1.0, 1.0),
                 periodic=(False, True, True), order=order)
    # drop the x-boundary ghosts: the neighbouring slabs stand behind those faces
    ni = m.n_interior
    keepf = (m.face_cells[:, 0] < ni) & (m.face_cells[:, 1] < ni)
    li = np.floor((m.cell_centroid[:ni, 0] - lo) / hx + 1e-9).astype(np.int64)
    kind = np.where((li >= halo) & (li < halo + nx), L.CELL_OWNED,
                    np.where((li == halo - 1) | (li == halo + nx), L.CELL_HALO, L.CELL_HALO_OUTER)).astype(np.uint8)
    core = kind != L.CELL_HALO_OUTER
    fc = m.face_cells[keepf]
    keepf2 = core[fc[:, 0]] | core[fc[:, 1]]
    fsel = np.nonzero(keepf)[0][keepf2]
    lm = Mesh(3, m.face_cells[fsel].copy(), m.face_normal[fsel].copy(), m.face_centroid[fsel].copy(), m.cell_centroid[:ni].copy(),
              m.cell_volume[:ni].copy(), kind, None if m.face_shift is None else m.face_shift[fsel].copy(),
              n_interior=int((kind == L.CELL_OWNED).sum()), shape=(nx, ny, nz))
    gi = np.mod(rank * nx - halo + li, nxg)
    j = np.floor(m.cell_centroid[:ni, 1] * ny).astype(np.int64)
    k = np.floor(m.cell_centroid[:ni, 2] * nz).astype(np.int64)
    return LocalDomain(lm, gi + nxg * (j + ny * k), (gi // nx).astype(np.int32), rank, nparts)


@dataclass
class ExchangePlan:
    """Per peer rank: the local rows to pack and send, and the local rows the received message fills,
    both in ascending global id (the order the two ends agree on)."""
    send: dict
    recv: dict

    @staticmethod
    def build(dom: LocalDomain, requests_to_me: dict) -> "ExchangePlan":
        """requests_to_me[p] = the global ids rank p needs from this rank (p's LocalDomain.needs()[rank])."""
        pos = {int(g): i for i, g in enumerate(dom.gid)}
        recv = {p: np.array([pos[int(g)] for g in gids], np.int32) for p, gids in dom.needs().items()}
        send = {}
        for p, gids in requests_to_me.items():
            rows = np.array([pos.get(int(g), -1) for g in np.sort(gids)], np.int32)
            if (rows < 0).any() or (dom.owner[rows] != dom.rank).any():
                raise ValueError(f"rank {p} asked rank {dom.rank} for cells it does not own")
            send[int(p)] = rows
        return ExchangePlan(send, recv)


def all_plans(domains: list) -> list:
    """The exchange plans of every rank when all local domains are at hand (one process)."""
    needs = [d.needs() for d in domains]
    return [ExchangePlan.build(d, {p: needs[p][d.rank] for p in range(len(domains)) if d.rank in needs[p]}) for d in domains]


def plan_with(dom: LocalDomain, group=None) -> ExchangePlan:
    """Build this rank's plan by exchanging the request lists with every other rank (set-up time)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = dom.needs()
    gathered = [None] * world
    dist.all_gather_object(gathered, {p: v.tolist() for p, v in mine.items()}, group=group)
    req = {p: np.asarray(gathered[p][dom.rank], np.int64) for p in range(world) if p != dom.rank and dom.rank in gathered[p]}
    return ExchangePlan.build(dom, req)


class HaloExchange:
    """Refresh a local state array (torch tensor on this rank's GPU, (n_local, width) FP64) from the
    owners of its non-owned rows: pack (abl_rows_gather), NCCL point-to-point, unpack (abl_rows_scatter),
    all ordered on the current CUDA stream."""

    def __init__(self, plan: ExchangePlan, width: int, device, group=None):
        import torch
        self.torch = torch
        self.group = group
        self.width = width
        self.device = device
        self.peers = sorted(set(plan.send) | set(plan.recv))
        self.send_idx = {p: torch.from_numpy(plan.send.get(p, np.zeros(0, np.int32))).to(device) for p in self.peers}
        self.recv_idx = {p: torch.from_numpy(plan.recv.get(p, np.zeros(0, np.int32))).to(device) for p in self.peers}
        self.send_buf = {p: torch.empty((self.send_idx[p].numel(), width), dtype=torch.float64, device=device) for p in self.peers}
        self.recv_buf = {p: torch.empty((self.recv_idx[p].numel(), width), dtype=torch.float64, device=device) for p in self.peers}
        self.bytes_per_exchange = sum(8 * width * (self.send_idx[p].numel() + self.recv_idx[p].numel()) for p in self.peers)

    def exchange(self, U):
        torch = self.torch
        import torch.distributed as dist
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for p in self.peers:
            n = self.send_idx[p].numel()
            if n:
                L.check(L.lib.abl_rows_gather(C.c_void_p(U.data_ptr()), self.width, C.c_void_p(self.send_idx[p].data_ptr()), n,
                                              C.c_void_p(self.send_buf[p].data_ptr()), C.c_void_p(stream)), "abl_rows_gather")
        ops = []
        for p in self.peers:
            if self.recv_idx[p].numel():
                ops.append(dist.P2POp(dist.irecv, self.recv_buf[p], p, group=self.group))
            if self.send_idx[p].numel():
                ops.append(dist.P2POp(dist.isend, self.send_buf[p], p, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for p in self.peers:
            n = self.recv_idx[p].numel()
            if n:
                L.check(L.lib.abl_rows_scatter(C.c_void_p(self.recv_buf[p].data_ptr()), self.width, C.c_void_p(self.recv_idx[p].data_ptr()),
                                               n, C.c_void_p(U.data_ptr()), C.c_void_p(stream)), "abl_rows_scatter")


    def exchange_adjoint(self, Ubar):
        """Transpose of exchange(): the adjoint held in this rank's halo rows goes back to their owners,
        which add it into the owned rows (peers in ascending order, a fixed summation order); the halo
        rows are cleared."""
        torch = self.torch
        import torch.distributed as dist
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for p in self.peers:
            n = self.recv_idx[p].numel()
            if n:
                L.check(L.lib.abl_rows_gather(C.c_void_p(Ubar.data_ptr()), self.width, C.c_void_p(self.recv_idx[p].data_ptr()), n,
                                              C.c_void_p(self.recv_buf[p].data_ptr()), C.c_void_p(stream)), "abl_rows_gather")
        ops = []
        for p in self.peers:
            if self.send_idx[p].numel():
                ops.append(dist.P2POp(dist.irecv, self.send_buf[p], p, group=self.group))
            if self.recv_idx[p].numel():
                ops.append(dist.P2POp(dist.isend, self.recv_buf[p], p, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for p in self.peers:
            n = self.send_idx[p].numel()
            if n:
                L.check(L.lib.abl_rows_scatter_add(C.c_void_p(self.send_buf[p].data_ptr()), self.width,
                                                   C.c_void_p(self.send_idx[p].data_ptr()), n, C.c_void_p(Ubar.data_ptr()),
                                                   C.c_void_p(stream)), "abl_rows_scatter_add")
        for p in self.peers:
            if self.recv_idx[p].numel():
                Ubar.index_fill_(0, self.recv_idx[p].long(), 0.0)


class DistributedRHS:
    """One rank's RHS of a partitioned mesh: the halo exchange, then the local RHS on the same stream
    (the order TimeStepper::SolverComputeRHSFunction runs DMGlobalToLocal and the RHS in)."""

    def __init__(self, dom: LocalDomain, eos, processes, petscfv_type: str, limiter: str, device: int = 0, group=None):
        import torch
        import torch.distributed as dist

        from . import fv
        self.torch = torch
        self.dom = dom
        self.solver = fv.FiniteVolumeSolver(dom.mesh, eos, processes, petscfv_type, limiter, device=device)
        self.device = torch.device("cuda", device)
        distributed = dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1
        plan = plan_with(dom, group) if distributed else ExchangePlan({}, {})
        self.halo = HaloExchange(plan, self.solver.nc, self.device, group)
        self.comm_stream = None  # created on the first overlapped exchange

    def ComputeRHSDevice(self, time: float, U, F, precision: int = L.PRECISION_FP64, overlap: bool = True):
        """F += RHS(U) on the owned rows after refreshing U's halo rows; U, F torch tensors on this GPU.

        With overlap, the exchange runs on a second stream while the current one computes the part of the
        RHS that reads no halo row (abl_fv_rhs_phase, interior phase); the rest follows once the exchange
        is done. The exchange writes only halo rows and the interior phase reads none, so the two overlap
        without a race, and the residual equals the serial order's bit for bit."""
        torch = self.torch
        cur = torch.cuda.current_stream(self.device)
        if not overlap or not self.halo.peers:
            self.halo.exchange(U)
            self.solver.ComputeRHSDevice(time, U.data_ptr(), F.data_ptr(), precision, cur.cuda_stream)
            return
        if self.comm_stream is None:
            self.comm_stream = torch.cuda.Stream(self.device)
        self.comm_stream.wait_stream(cur)  # U is written before the exchange packs it
        with torch.cuda.stream(self.comm_stream):
            self.halo.exchange(U)
        self.solver.ComputeRHSPhaseDevice(time, U.data_ptr(), F.data_ptr(), L.RHS_PHASE_INTERIOR, precision, cur.cuda_stream)
        cur.wait_stream(self.comm_stream)
        self.solver.ComputeRHSPhaseDevice(time, U.data_ptr(), F.data_ptr(), L.RHS_PHASE_REST, precision, cur.cuda_stream)

    def ComputeJVPDevice(self, time: float, U, dU, dF, F=None):
        """dF += J(U) dU on the owned rows (and F += RHS(U) when F is given), after refreshing the halo
        rows of both U and dU."""
        self.halo.exchange(U)
        self.halo.exchange(dU)
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        self.solver.ComputeJVPDevice(time, U.data_ptr(), dU.data_ptr(), dF.data_ptr(), F.data_ptr() if F is not None else 0, stream)

    def ComputeVJPDevice(self, time: float, U, Fbar, Ubar):
        """Ubar += J(U)^T Fbar for the owned rows of the whole partitioned problem: the local adjoint, then
        the halo rows' share sent back to their owners (exchange_adjoint; Ubar's halo rows are consumed)."""
        self.halo.exchange(U)
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        self.solver.ComputeVJPDevice(time, U.data_ptr(), Fbar.data_ptr(), Ubar.data_ptr(), stream)
        self.halo.exchange_adjoint(Ubar)

    def close(self):
        self.solver.close()
