"""Partitioned RHS on the CPU: cell partition, two-layer halo, exchange plans (ablate_b200.distributed).

The oracle RHS evaluated on every rank's local mesh, after the halo rows were filled through the
exchange plans, must reproduce the single-domain oracle RHS on the owned cells: the partitioned
evaluation of FiniteVolumeSolver::ComputeRHSFunction under MPI (DMGlobalToLocal before the RHS,
src/solver/timeStepper.cpp:343-344). The last tests run the exchange over torch.distributed with the
gloo backend and two ranks, for a Morton partition of a small mesh and for the bench's x-slabs.
"""
import os
import socket

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import distributed as D
from ablate_b200 import workloads
from ablate_b200.mesh import box_mesh
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R

CASES = ["tgv3d_ausmpup_lsq_minmod_visc", "sod2d_ausm_upwind", "box2d_ausmpup_vanleer_suth", "species3d_ns5", "pgspecies3d_ns2",
         "tets3d_pg_minmod"]


def _exchange_numpy(domains, plans, U_local):
    """Move the rows every plan names (what HaloExchange does with NCCL)."""
    msgs = {}
    for d, pl in zip(domains, plans):
        for p, rows in pl.send.items():
            msgs[(d.rank, p)] = U_local[d.rank][rows].copy()
    for d, pl in zip(domains, plans):
        for p, rows in pl.recv.items():
            U_local[d.rank][rows] = msgs[(p, d.rank)]


def _local_states(w, domains):
    # each rank starts with only the rows it owns (owned cells and its own ghosts); NaN elsewhere
    out = []
    for d in domains:
        U = np.full((d.mesh.n_cells, w.U.shape[1]), np.nan)
        mine = d.owner == d.rank
        U[mine] = w.U[d.gid[mine]]
        out.append(U)
    return out


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_oracle_rhs_equals_single_domain(name, nparts):
    w = R.case(name)
    phys, keep = w.physics()
    F_ref, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    part = D.partition_cells(w.mesh, nparts)
    assert (part >= 0).all() and set(np.unique(part)) == set(range(nparts))
    domains = [D.submesh(w.mesh, part, r) for r in range(nparts)]
    # every interior cell is owned exactly once
    owned_g = np.concatenate([d.gid[d.owned] for d in domains])
    assert np.array_equal(np.sort(owned_g), np.nonzero(w.mesh.cell_kind != L.CELL_BOUNDARY)[0])
    plans = D.all_plans(domains)
    U_local = _local_states(w, domains)
    _exchange_numpy(domains, plans, U_local)
    aux_g = initial_aux(w)
    for d, U in zip(domains, U_local):
        assert np.array_equal(U, w.U[d.gid])  # the exchange filled every row with its owner's value
        F, _ = orc.rhs(d.mesh, phys, U, aux_g[d.gid])
        o = d.owned
        # local meshes keep the global face order: the owned rows agree bit for bit
        np.testing.assert_array_equal(F[o], F_ref[d.gid[o]])


@pytest.mark.parametrize("nparts", [2, 4])
def test_slab_domains_reproduce_the_periodic_box(nparts):
    shape = (8, 4, 4)
    g = box_mesh(shape, periodic=(True, True, True))
    st = workloads.tgv_state(g)
    w = workloads.tgv3d(8)
    phys, keep = w.physics()
    F_ref, _ = orc.rhs(g, phys, st, None)
    domains = [D.slab_domain(shape, nparts, r) for r in range(nparts)]
    for d in domains:
        # geometry of every local cell is its global cell's (up to the periodic image in x)
        dx = np.mod(d.mesh.cell_centroid - g.cell_centroid[d.gid] + 0.5, 1.0) - 0.5
        assert np.abs(dx).max() < 1e-12
        assert d.owned.sum() == np.prod(shape) // nparts
    plans = D.all_plans(domains)
    U_local = [np.where((d.owner == d.rank)[:, None], st[d.gid], np.nan) for d in domains]
    _exchange_numpy(domains, plans, U_local)
    for d, U in zip(domains, U_local):
        assert np.array_equal(U, st[d.gid])
        F, _ = orc.rhs(d.mesh, phys, U, None)
        o = d.owned
        # a slab numbers its faces differently from the global box: least-squares weights and sums
        # may round differently
        err = np.linalg.norm(F[o] - F_ref[d.gid[o]]) / np.linalg.norm(F_ref[d.gid[o]])
        assert err < 1e-12, err


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, name, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if name == "slab":
            # the bench's layout: slabs of the periodic box built per rank, plans from the gathered requests
            shape = (8, 4, 4)
            g = box_mesh(shape, periodic=(True, True, True))
            w = workloads.tgv3d(8)
            w.mesh, w.U = g, workloads.tgv_state(g)
            d = D.slab_domain(shape, world, rank)
        else:
            w = R.case(name)
            part = D.partition_cells(w.mesh, world)
            d = D.submesh(w.mesh, part, rank)
        phys, keep = w.physics()
        plan = D.plan_with(d)
        U = np.full((d.mesh.n_cells, w.U.shape[1]), np.nan)
        mine = d.owner == rank
        U[mine] = w.U[d.gid[mine]]
        ops, bufs = [], {}
        for p in sorted(set(plan.send) | set(plan.recv)):
            if p in plan.recv:
                bufs[p] = torch.empty((plan.recv[p].size, U.shape[1]), dtype=torch.float64)
                ops.append(dist.P2POp(dist.irecv, bufs[p], p))
            if p in plan.send:
                ops.append(dist.P2POp(dist.isend, torch.from_numpy(np.ascontiguousarray(U[plan.send[p]])), p))
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        for p, b in bufs.items():
            U[plan.recv[p]] = b.numpy()
        F, _ = orc.rhs(d.mesh, phys, U, initial_aux(w)[d.gid])
        got = [None] * world
        dist.all_gather_object(got, (d.gid[d.owned], F[d.owned], bool(np.array_equal(U, w.U[d.gid]))))
        if rank == 0:
            F_ref, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
            if name == "slab":  # face numbering differs from the global box: agreement to rounding
                same = all(np.linalg.norm(f - F_ref[g]) <= 1e-12 * np.linalg.norm(F_ref[g]) for g, f, _ in got)
            else:
                same = all(np.array_equal(f, F_ref[g]) for g, f, _ in got)
            ok = all(x[2] for x in got) and same
            cover = np.sort(np.concatenate([g for g, _, _ in got]))
            ok = ok and np.array_equal(cover, np.nonzero(w.mesh.cell_kind != L.CELL_BOUNDARY)[0])
            q.put(ok)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "sod2d_ausm_upwind", "slab"])
def test_two_gloo_ranks_exchange_halos_and_match_the_single_domain(name):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, name, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert q.get(timeout=5) is True


def _exchange_adjoint_numpy(domains, plans, Ub_local):
    """Transpose of _exchange_numpy: each halo row's adjoint is added into its owner's row (peers in
    ascending order) and cleared, as HaloExchange.exchange_adjoint does with NCCL."""
    msgs = {}
    for d, pl in zip(domains, plans):
        for p, rows in pl.recv.items():
            msgs[(d.rank, p)] = Ub_local[d.rank][rows].copy()
    for d, pl in zip(domains, plans):
        for p in sorted(pl.send):
            Ub_local[d.rank][pl.send[p]] += msgs[(p, d.rank)]
    for d, pl in zip(domains, plans):
        for p, rows in pl.recv.items():
            Ub_local[d.rank][rows] = 0.0


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "tets3d_pg_minmod"])
def test_transposed_exchange_is_the_adjoint_of_the_exchange(name):
    """<E x, y> = <x, E^T y>: E fills every local row from the owned rows of x (the halo exchange), E^T
    adds the halo rows of y into their owners; x lives on the owned rows, y on all local rows."""
    w = R.case(name)
    part = D.partition_cells(w.mesh, 3)
    domains = [D.submesh(w.mesh, part, r) for r in range(3)]
    plans = D.all_plans(domains)
    rng = np.random.default_rng(6)
    nc = w.U.shape[1]
    xg = rng.standard_normal((w.mesh.n_cells, nc))
    X = []
    for d in domains:
        a = np.zeros((d.mesh.n_cells, nc))
        mine = d.owner == d.rank
        a[mine] = xg[d.gid[mine]]
        X.append(a)
    _exchange_numpy(domains, plans, X)
    Y = [rng.standard_normal((d.mesh.n_cells, nc)) for d in domains]
    # only the rows the exchange fills carry the pairing: owned rows and exchanged halo rows
    lhs = 0.0
    for d, pl, x, y in zip(domains, plans, X, Y):
        mine = d.owner == d.rank
        rows = np.concatenate([np.nonzero(mine)[0]] + [r for r in pl.recv.values()])
        lhs += float(np.sum(x[rows] * y[rows]))
    Yt = [y.copy() for y in Y]
    _exchange_adjoint_numpy(domains, plans, Yt)
    rhs = 0.0
    for d, x, yt in zip(domains, X, Yt):
        mine = d.owner == d.rank
        rhs += float(np.sum(x[mine] * yt[mine]))
    assert abs(lhs - rhs) <= 1e-12 * sum(float(np.abs(y).sum()) for y in Y)
