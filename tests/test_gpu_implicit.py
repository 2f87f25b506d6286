"""Matrix-free BDF1/BDF2 with Newton-GMRES(30) on the device JVP (ablate_b200.implicit): the step solves
its nonlinear system, and BDF2 converges at second order against a fine SSP-RK3 march. These run the
wall-bounded channel with unlimited least-squares gradients: Newton needs a differentiable residual, and
a limited scheme is not (the limiter's branches and the minimising face switch under the Newton
updates; the bench reports how far Newton gets there)."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from ablate_b200.implicit import BDFStepper
from oracle import stepper as S

pytestmark = pytest.mark.gpu


def _setup(n=10):
    w = workloads.wall3d(n)
    w.limiter = "none"
    phys, keep = w.physics()
    s = w.solver()
    s.SetBoundary(*w.boundary)
    dt = 0.5 * S.cfl_dt(w.mesh, phys, w.U, 1.0)
    return w, s, dt


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausmpup_vanleer_suth"])
def test_frozen_limiter_tangent(name):
    """The frozen-limiter tangent is linear in the direction, differs from the exact one only through
    the limiter factor's derivative, and leaves the exact mode (and the VJP) untouched."""
    torch = pytest.importorskip("torch")
    from tests import rhs_cases as R
    w = R.case(name)
    s = w.solver()
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(3)
    U = torch.from_numpy(w.U).to(dev)
    a = torch.from_numpy(rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)).to(dev)
    b = torch.from_numpy(rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)).to(dev)

    def jvp(v):
        dF = torch.zeros_like(U)
        s.ComputeJVPDevice(0.0, U.data_ptr(), v.data_ptr(), dF.data_ptr(), 0, st)
        return dF

    exact = jvp(a)
    s.SetJVPMode(L.JVP_FROZEN_LIMITER)
    fa, fb, fab = jvp(a), jvp(b), jvp(2.0 * a - 3.0 * b)
    s.SetJVPMode(L.JVP_EXACT)
    assert torch.equal(jvp(a), exact)
    assert float((fab - (2.0 * fa - 3.0 * fb)).norm()) <= 1e-12 * float(fab.norm())
    assert float((fa - exact).norm()) > 1e-6 * float(exact.norm())  # the limiter is active here


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
    n = 4  # march over 4 CFL-0.5 steps, at 1/2, 1/4 and 1/8 of that step
    ref = U0.clone()
    for _ in range(n * 64):
        s.StepDevice(L.STEP_SSPRK3, 0.0, dt / 64, ref.data_ptr(), L.PRECISION_FP64, st)
    errs = []
    for m in (2, 4, 8):
        bdf = BDFStepper(s, dt / m, snes_rtol=1e-10, ksp_rtol=1e-8)
        X = U0.clone()
        for _ in range(n * m):
            bdf.step(X)
        errs.append(float((X[owned] - ref[owned]).norm()))
        assert bdf.stats["snes_unconverged"] == 0
    assert s.Status() == L.OK
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    # the BDF1 start adds a second-order term with a large constant: the order approaches 2 from below
    assert orders[-1] >= 1.75 and orders[-1] <= 2.3 and orders[-1] >= orders[0] - 0.05, (errs, orders)
