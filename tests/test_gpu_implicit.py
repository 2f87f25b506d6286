"""Matrix-free BDF1/BDF2 with Newton-GMRES(30) on the device JVP (ablate_b200.implicit): the step solves
its nonlinear system, and BDF2 converges at second order against a fine SSP-RK3 march."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from ablate_b200.implicit import BDFStepper
from oracle import stepper as S

pytestmark = pytest.mark.gpu


def _setup(n=10):
    w = workloads.wall3d(n)
    phys, keep = w.physics()
    s = w.solver()
    s.SetBoundary(*w.boundary)
    dt = 0.5 * S.cfl_dt(w.mesh, phys, w.U, 1.0)
    return w, s, dt


def test_bdf_steps_solve_their_nonlinear_system():
    torch = pytest.importorskip("torch")
    w, s, dt = _setup()
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    U = torch.from_numpy(w.U).to(dev)
    s.FillGhostsDevice(U.data_ptr(), st)
    owned = torch.from_numpy(w.mesh.cell_kind == L.CELL_OWNED).to(dev)[:, None]
    bdf = BDFStepper(s, 4 * dt)
    hist = [U.clone()]
    for _ in range(3):
        bdf.step(U)
        hist.append(U.clone())
    assert s.Status() == L.OK
    assert bdf.stats["steps"] == 3 and bdf.stats["newton"] >= 3
    # independent residuals: BDF1 then BDF2
    for k, (a1, a2, beta) in enumerate([(1.0, 0.0, 1.0), (4 / 3, -1 / 3, 2 / 3), (4 / 3, -1 / 3, 2 / 3)]):
        X = hist[k + 1].clone()
        F = torch.zeros_like(X)
        s.ComputeRHSDevice(0.0, X.data_ptr(), F.data_ptr(), L.PRECISION_FP64, st)
        R = X - a1 * hist[k] - (a2 * hist[k - 1] if k > 0 else 0.0) - beta * 4 * dt * F
        scale = float((beta * 4 * dt * F * owned).norm())
        assert float((R * owned).norm()) <= 1e-6 * scale, k


def test_bdf2_is_second_order():
    torch = pytest.importorskip("torch")
    w, s, dt = _setup()
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    U0 = torch.from_numpy(w.U).to(dev)
    s.FillGhostsDevice(U0.data_ptr(), st)
    owned = torch.from_numpy(w.mesh.cell_kind == L.CELL_OWNED).to(dev)
    n = 8
    ref = U0.clone()
    for _ in range(n * 16):
        s.StepDevice(L.STEP_SSPRK3, 0.0, dt / 16, ref.data_ptr(), L.PRECISION_FP64, st)
    errs = []
    for m in (1, 2):
        bdf = BDFStepper(s, dt / m, snes_rtol=1e-10, ksp_rtol=1e-8)
        X = U0.clone()
        for _ in range(n * m):
            bdf.step(X)
        errs.append(float((X[owned] - ref[owned]).norm()))
    assert s.Status() == L.OK
    order = np.log2(errs[0] / errs[1])
    assert 1.6 <= order <= 2.6, (errs, order)
