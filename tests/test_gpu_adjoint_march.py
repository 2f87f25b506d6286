"""Gradients of the wall-pressure functional of a marched state on the device (ablate_b200.adjoint):
the ghost-fill tangent and transpose against the oracle's, the functional and its state gradient against
the oracle's, the adjoint march against the tangent march (dot-product test), and the gradients with
respect to the initial state and the inlet speed against central differences (eps 1e-7 relative) of
the device march and of the oracle's march."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from ablate_b200.adjoint import ExplicitMarch, functional_gradient, inlet_state
from oracle import stepper as S
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.device("cuda", 0))


def _st(torch):
    return torch.cuda.current_stream().cuda_stream


def _tables(w):
    ref = np.abs(w.U[w.mesh.cell_kind == L.CELL_OWNED]).mean(0)
    return [(S.OUTFLOW, None, False), (S.DIRICHLET, list(ref * 1.1), False), (S.DIRICHLET, list(ref * 0.9), True),
            (S.SLIP_WALL, None, False), (S.NOSLIP_WALL, None, False)]


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "box2d_ausmpup_vanleer_suth", "species3d_ns5", "box1d_riemann_upwind"])
def test_fill_tangent_and_transpose_match_the_oracle(name):
    torch = pytest.importorskip("torch")
    w = R.case(name)
    s = w.solver()
    rng = np.random.default_rng(7)
    table = _tables(w)
    cell_bc = rng.integers(0, len(table), w.mesh.n_cells).astype(np.int32)
    s.SetBoundary(table, cell_bc)
    dU = rng.standard_normal(w.U.shape)
    d = _dev(torch, dU)
    s.FillGhostsJVPDevice(d.data_ptr(), _st(torch))
    np.testing.assert_array_equal(d.cpu().numpy(), S.fill_ghosts_tangent(w.mesh, dU.copy(), table, cell_bc))
    lam = rng.standard_normal(w.U.shape)
    lb = _dev(torch, lam)
    vb = s.FillGhostsVJPDevice(lb.data_ptr(), _st(torch))
    ref, vref = S.fill_ghosts_adjoint(w.mesh, lam.copy(), table, cell_bc)
    np.testing.assert_array_equal(lb.cpu().numpy(), ref)
    nc = w.U.shape[1]
    np.testing.assert_allclose(vb[:, :nc], vref, rtol=1e-13, atol=1e-13 * np.abs(vref).max())
    assert np.all(vb[:, nc:] == 0.0)


@pytest.mark.parametrize("name", ["wall3d", "species3d_ns5"])
def test_pressure_functional_matches_the_oracle(name):
    torch = pytest.importorskip("torch")
    if name == "wall3d":
        w = workloads.wall3d(8)
        cells, wts = w.functional
    else:
        w = R.case(name)
        owned = np.nonzero(w.mesh.cell_kind == L.CELL_OWNED)[0]
        cells, wts = owned[::3], np.linspace(0.5, 1.5, owned[::3].size)
    phys, keep = w.physics()
    s = w.solver()
    s.SetPressureFunctional(cells, wts)
    U = _dev(torch, w.U)
    G = torch.zeros_like(U)
    J = s.PressureFunctionalDevice(U.data_ptr(), G.data_ptr(), _st(torch))
    assert s.Status() == L.OK
    gamma = 1.4 if name == "wall3d" else None
    Jr, Gr = S.pressure_functional(w.mesh, phys, w.U, cells, wts, gamma=gamma)
    assert abs(J - Jr) <= 1e-13 * abs(Jr)
    g = G.cpu().numpy()
    if Gr is not None:
        np.testing.assert_allclose(g, Gr, rtol=1e-13, atol=1e-13 * np.abs(Gr).max())
    else:
        # mixture EOS: the gradient against central differences of the oracle's functional
        rng = np.random.default_rng(1)
        for _ in range(3):
            d = np.zeros_like(w.U)
            d[cells] = rng.standard_normal((cells.size, w.U.shape[1])) * np.abs(w.U[cells])
            eps = 1e-6
            fd = (S.pressure_functional(w.mesh, phys, w.U + eps * d, cells, wts)[0]
                  - S.pressure_functional(w.mesh, phys, w.U - eps * d, cells, wts)[0]) / (2 * eps)
            assert abs(fd - float(np.sum(g * d))) <= 1e-6 * abs(fd), (fd, float(np.sum(g * d)))


def _wall_case(n):
    w = workloads.wall3d(n)
    phys, keep = w.physics()
    s = w.solver()
    table, cell_bc = w.boundary
    s.SetBoundary(table, cell_bc)
    s.SetPressureFunctional(*w.functional)
    dt = 0.4 * S.cfl_dt(w.mesh, phys, w.U, 1.0)
    return w, phys, keep, s, dt


@pytest.mark.parametrize("scheme", [L.STEP_EULER, L.STEP_SSPRK3])
def test_adjoint_march_is_the_transpose_of_the_tangent_march(scheme):
    torch = pytest.importorskip("torch")
    w, phys, keep, s, dt = _wall_case(10)
    m = ExplicitMarch(s, scheme, dt, 4)
    U0 = _dev(torch, w.U)
    J, lam0, vbar = functional_gradient(s, m, U0)
    assert s.Status() == L.OK
    rng = np.random.default_rng(11)
    owned = (w.mesh.cell_kind == L.CELL_OWNED)[:, None]
    dU0 = _dev(torch, np.where(owned, rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0), 0.0))
    UK, dUK = m.tangent(U0, dU0)
    g = torch.zeros_like(UK)
    s.PressureFunctionalDevice(UK.data_ptr(), g.data_ptr(), _st(torch))
    lhs = float((g * dUK).sum())
    rhs = float((lam0 * dU0).sum())
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), float((lam0 * dU0).abs().sum())), (lhs, rhs)
    # the tangent march's state is the forward march's (the dual numbers' values round like the RHS's
    # up to the FP64 reciprocal's last bit)
    UF = m.forward(U0, keep=False)
    assert float((UK - UF).norm()) <= 1e-13 * float(UF.norm())


def test_functional_gradients_match_central_differences():
    torch = pytest.importorskip("torch")
    w, phys, keep, s, dt = _wall_case(10)
    K = 4
    m = ExplicitMarch(s, L.STEP_SSPRK3, dt, K)
    U0 = _dev(torch, w.U)
    J, lam0, vbar = functional_gradient(s, m, U0)
    table, cell_bc = w.boundary
    cells, wts = w.functional
    rho0, p0 = 101325.0 / (287.0 * 300.0), 101325.0
    V = 0.3 * np.sqrt(1.4 * 287.0 * 300.0)
    value, dvalue = inlet_state(rho0, p0, V, (1.0, 0.0, 0.0))
    dJdV = float(np.dot(vbar[0, :5], dvalue))

    def J_at(speed, U, device=True):
        v, _ = inlet_state(rho0, p0, speed, (1.0, 0.0, 0.0))
        tb = [(L.BC_DIRICHLET, list(v), False)] + list(table[1:])
        if not device:
            return S.march_functional(w.mesh, phys, U, dt, K, tb, cell_bc, cells, wts)
        s.SetBoundary(tb, cell_bc)
        Uk = m.forward(_dev(torch, U), keep=False)
        out = s.PressureFunctionalDevice(Uk.data_ptr(), 0, _st(torch))
        s.SetBoundary(table, cell_bc)
        return out

    # the functional itself agrees with the oracle's march
    assert abs(J - J_at(V, w.U, device=False)) <= 1e-12 * abs(J)
    h = 1e-7 * V
    fd_dev = (J_at(V + h, w.U) - J_at(V - h, w.U)) / (2 * h)
    fd_or = (J_at(V + h, w.U, False) - J_at(V - h, w.U, False)) / (2 * h)
    assert abs(dJdV) > 0
    assert abs(fd_dev - dJdV) <= 1e-5 * abs(dJdV), (fd_dev, dJdV)
    assert abs(fd_or - dJdV) <= 1e-5 * abs(dJdV), (fd_or, dJdV)
    # initial-state gradient along smooth seeded directions. The limited scheme has kinks (limiter
    # branches, the minimising face) a relative perturbation of 1e-7 of white noise already crosses in
    # some cells; a smooth direction at eps 1e-8 stays on one branch.
    owned = (w.mesh.cell_kind == L.CELL_OWNED)[:, None]
    x = w.mesh.cell_centroid
    lam = lam0.cpu().numpy()
    rng = np.random.default_rng(12)
    for _ in range(2):
        k = rng.uniform(1.0, 3.0, 3)
        ph = rng.uniform(0.0, 2 * np.pi, (w.U.shape[1], 3))
        d = np.stack([np.sin(2 * np.pi * k[0] * x[:, 0] + ph[c, 0]) * np.sin(2 * np.pi * k[1] * x[:, 1] + ph[c, 1])
                      * np.cos(2 * np.pi * k[2] * x[:, 2] + ph[c, 2]) for c in range(w.U.shape[1])], 1)
        d = np.where(owned, d * np.abs(w.U).mean(0), 0.0)
        eps = 1e-8
        fd = (J_at(V, w.U + eps * d) - J_at(V, w.U - eps * d)) / (2 * eps)
        ad = float(np.sum(lam * d))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
