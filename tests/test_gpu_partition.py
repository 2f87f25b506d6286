"""Partitioned device RHS on one GPU: every rank's local mesh gets its own solver, the halo rows move
through the exchange kernels (abl_rows_gather into a message buffer, abl_rows_scatter out of it; the
buffer copy stands in for the NCCL transfer), and the owned rows of the local residuals must equal the
single-domain device residual bit for bit."""
import ctypes as C

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import distributed as D
from ablate_b200 import fv
from ablate_b200.workloads import initial_aux
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu


def _rows(torch, fn, src, idx, dst):
    s = torch.cuda.current_stream()
    L.check(getattr(L.lib, fn)(C.c_void_p(src.data_ptr()), src.shape[1], C.c_void_p(idx.data_ptr()), idx.numel(),
                               C.c_void_p(dst.data_ptr()), C.c_void_p(s.cuda_stream)), fn)


def test_row_gather_and_scatter_kernels():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    for width in (1, 4, 5, 14):
        src = torch.from_numpy(rng.standard_normal((1000, width))).to(dev)
        idx_np = rng.permutation(1000)[:377].astype(np.int32)
        idx = torch.from_numpy(idx_np).to(dev)
        buf = torch.empty((377, width), dtype=torch.float64, device=dev)
        _rows(torch, "abl_rows_gather", src, idx, buf)
        np.testing.assert_array_equal(buf.cpu().numpy(), src.cpu().numpy()[idx_np])
        dst = torch.zeros_like(src)
        _rows(torch, "abl_rows_scatter", buf, idx, dst)
        ref = np.zeros((1000, width))
        ref[idx_np] = src.cpu().numpy()[idx_np]
        np.testing.assert_array_equal(dst.cpu().numpy(), ref)


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "sod2d_ausm_upwind", "species3d_ns5", "box2d_ausmpup_vanleer_suth",
                                  "tets3d_ns9"])
@pytest.mark.parametrize("precision", [L.PRECISION_FP64, L.PRECISION_MIXED])
def test_partitioned_device_rhs_equals_single_domain(name, precision):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    w = R.case(name)
    s = w.solver()
    aux_g = initial_aux(w)
    s.SetAux(aux_g)
    F_ref = np.zeros_like(w.U)
    s.ComputeRHSFunction(0.0, w.U, F_ref, precision)
    nparts = 3
    part = D.partition_cells(w.mesh, nparts)
    doms = [D.submesh(w.mesh, part, r) for r in range(nparts)]
    plans = D.all_plans(doms)
    solvers, U = [], []
    for d in doms:
        sv = fv.FiniteVolumeSolver(d.mesh, w.eos, w.processes, w.petscfv_type, w.limiter)
        sv.SetAux(aux_g[d.gid])
        solvers.append(sv)
        u = np.full((d.mesh.n_cells, w.U.shape[1]), np.nan)
        mine = d.owner == d.rank
        u[mine] = w.U[d.gid[mine]]
        U.append(torch.from_numpy(u).to(dev))
    # exchange: pack at the owner, unpack at the receiver
    for d, pl in zip(doms, plans):
        for p, rows in pl.recv.items():
            send_rows = torch.from_numpy(plans[p].send[d.rank]).to(dev)
            buf = torch.empty((send_rows.numel(), w.U.shape[1]), dtype=torch.float64, device=dev)
            _rows(torch, "abl_rows_gather", U[p], send_rows, buf)
            _rows(torch, "abl_rows_scatter", buf, torch.from_numpy(rows).to(dev), U[d.rank])
    for d, sv, u in zip(doms, solvers, U):
        assert np.array_equal(u.cpu().numpy(), w.U[d.gid])
        F = torch.zeros_like(u)
        sv.ComputeRHSDevice(0.0, u.data_ptr(), F.data_ptr(), precision, torch.cuda.current_stream().cuda_stream)
        assert sv.Status() == L.OK
        o = d.owned
        np.testing.assert_array_equal(F.cpu().numpy()[o], F_ref[d.gid[o]])
        sv.close()


def test_row_scatter_add_kernel():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(4)
    for width in (1, 5, 14):
        base = rng.standard_normal((500, width))
        src = torch.from_numpy(rng.standard_normal((123, width))).to(dev)
        idx_np = rng.permutation(500)[:123].astype(np.int32)
        dst = torch.from_numpy(base.copy()).to(dev)
        _rows(torch, "abl_rows_scatter_add", src, torch.from_numpy(idx_np).to(dev), dst)
        ref = base.copy()
        ref[idx_np] += src.cpu().numpy()
        np.testing.assert_array_equal(dst.cpu().numpy(), ref)


def _partitioned(torch, w, nparts, dev):
    aux_g = initial_aux(w)
    part = D.partition_cells(w.mesh, nparts)
    doms = [D.submesh(w.mesh, part, r) for r in range(nparts)]
    plans = D.all_plans(doms)
    solvers = []
    for d in doms:
        sv = fv.FiniteVolumeSolver(d.mesh, w.eos, w.processes, w.petscfv_type, w.limiter)
        sv.SetAux(aux_g[d.gid])
        solvers.append(sv)
    return doms, plans, solvers


def _exchange(torch, doms, plans, arrays, dev, width):
    for d, pl in zip(doms, plans):
        for p, rows in pl.recv.items():
            send_rows = torch.from_numpy(plans[p].send[d.rank]).to(dev)
            buf = torch.empty((send_rows.numel(), width), dtype=torch.float64, device=dev)
            _rows(torch, "abl_rows_gather", arrays[p], send_rows, buf)
            _rows(torch, "abl_rows_scatter", buf, torch.from_numpy(rows).to(dev), arrays[d.rank])


def _local(torch, doms, glob, dev, nan_halo=True):
    out = []
    for d in doms:
        a = np.full((d.mesh.n_cells, glob.shape[1]), np.nan if nan_halo else 0.0)
        mine = d.owner == d.rank
        a[mine] = glob[d.gid[mine]]
        out.append(torch.from_numpy(a).to(dev))
    return out


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausmpup_vanleer_suth", "species3d_ns5"])
def test_partitioned_jvp_and_vjp_equal_single_domain(name):
    """Tangent: halo rows of U and dU refreshed, local JVP; owned rows equal the single domain's bit for
    bit. Adjoint: local VJP, then every halo row's adjoint added into its owner's row (the transposed
    exchange, abl_rows_scatter_add); the assembled owned rows equal the single domain's VJP."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    w = R.case(name)
    s = w.solver()
    s.SetAux(initial_aux(w))
    rng = np.random.default_rng(8)
    dU = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)
    Fb = rng.standard_normal(w.U.shape)
    Ug, dUg, Fbg = (torch.from_numpy(a).to(dev) for a in (w.U, dU, Fb))
    dF_ref, Ub_ref = torch.zeros_like(Ug), torch.zeros_like(Ug)
    s.ComputeJVPDevice(0.0, Ug.data_ptr(), dUg.data_ptr(), dF_ref.data_ptr(), 0, st)
    s.ComputeVJPDevice(0.0, Ug.data_ptr(), Fbg.data_ptr(), Ub_ref.data_ptr(), st)
    dF_ref, Ub_ref = dF_ref.cpu().numpy(), Ub_ref.cpu().numpy()
    doms, plans, solvers = _partitioned(torch, w, 3, dev)
    nc = w.U.shape[1]
    U = _local(torch, doms, w.U, dev)
    dUl = _local(torch, doms, dU, dev)
    _exchange(torch, doms, plans, U, dev, nc)
    _exchange(torch, doms, plans, dUl, dev, nc)
    # every local Fbar row the residual reads is an owned row: the owner's Fbar
    Fbl = _local(torch, doms, Fb, dev, nan_halo=False)
    Ub = [torch.zeros_like(u) for u in U]
    for d, sv, u, du, fbl, ub in zip(doms, solvers, U, dUl, Fbl, Ub):
        dF = torch.zeros_like(u)
        sv.ComputeJVPDevice(0.0, u.data_ptr(), du.data_ptr(), dF.data_ptr(), 0, st)
        np.testing.assert_array_equal(dF.cpu().numpy()[d.owned], dF_ref[d.gid[d.owned]])
        sv.ComputeVJPDevice(0.0, u.data_ptr(), fbl.data_ptr(), ub.data_ptr(), st)
        assert sv.Status() == L.OK
    # transposed exchange: halo rows' adjoints back to the owners, peers in ascending order
    for d, pl in zip(doms, plans):
        for p in sorted(plans[d.rank].send):
            send_rows = torch.from_numpy(plans[d.rank].send[p]).to(dev)
            halo_rows = torch.from_numpy(plans[p].recv[d.rank]).to(dev)
            buf = torch.empty((halo_rows.numel(), nc), dtype=torch.float64, device=dev)
            _rows(torch, "abl_rows_gather", Ub[p], halo_rows, buf)
            _rows(torch, "abl_rows_scatter_add", buf, send_rows, Ub[d.rank])
    for d, ub in zip(doms, Ub):
        got = ub.cpu().numpy()[d.owned]
        ref = Ub_ref[d.gid[d.owned]]
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
    for sv in solvers:
        sv.close()


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "species3d_ns5", "tets3d_ns9", "species3d_ns4"])
def test_split_rhs_reads_no_halo_row_before_the_exchange(name):
    """abl_fv_rhs_phase: the interior phase runs while the halo rows still hold NaN (the exchange in
    flight), the rest after they are written; the owned residual equals the one-call RHS bit for bit."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    w = R.case(name)
    aux_g = initial_aux(w)
    nparts = 3
    part = D.partition_cells(w.mesh, nparts)
    doms = [D.submesh(w.mesh, part, r) for r in range(nparts)]
    stream = torch.cuda.current_stream().cuda_stream
    for d in doms:
        sv = fv.FiniteVolumeSolver(d.mesh, w.eos, w.processes, w.petscfv_type, w.limiter)
        full = torch.from_numpy(np.ascontiguousarray(w.U[d.gid])).to(dev)
        sv.SetAux(aux_g[d.gid])
        F_one = torch.zeros_like(full)
        sv.ComputeRHSDevice(0.0, full.data_ptr(), F_one.data_ptr(), L.PRECISION_FP64, stream)
        sv.SetAux(aux_g[d.gid])
        halo = torch.from_numpy(d.owner != d.rank).to(dev) & torch.from_numpy(d.mesh.cell_kind != L.CELL_BOUNDARY).to(dev)
        U = full.clone()
        U[halo] = float("nan")
        F = torch.zeros_like(full)
        sv.ComputeRHSPhaseDevice(0.0, U.data_ptr(), F.data_ptr(), L.RHS_PHASE_INTERIOR, L.PRECISION_FP64, stream)
        U[halo] = full[halo]  # the exchange arrives
        sv.ComputeRHSPhaseDevice(0.0, U.data_ptr(), F.data_ptr(), L.RHS_PHASE_REST, L.PRECISION_FP64, stream)
        torch.cuda.synchronize()
        assert sv.Status() == L.OK
        o = torch.from_numpy(d.owned).to(dev)
        assert torch.equal(F[o], F_one[o]), (name, d.rank)
        sv.close()
