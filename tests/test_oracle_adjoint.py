"""The oracle's ghost-fill derivative and its transpose, and the pressure functional's gradient (the
checkers of the device adjoint march, tests/test_gpu_adjoint_march.py), on the CPU."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from oracle import stepper as S
from tests import rhs_cases as R


def _tables(w):
    ref = np.abs(w.U[w.mesh.cell_kind == L.CELL_OWNED]).mean(0)
    return [(S.OUTFLOW, None, False), (S.DIRICHLET, list(ref * 1.1), False), (S.DIRICHLET, list(ref * 0.9), True),
            (S.SLIP_WALL, None, False), (S.NOSLIP_WALL, None, False)]


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "box2d_ausmpup_vanleer_suth", "species3d_ns5"])
def test_fill_adjoint_is_the_transpose_of_the_fill_tangent(name):
    w = R.case(name)
    rng = np.random.default_rng(3)
    table = _tables(w)
    cell_bc = rng.integers(0, len(table), w.mesh.n_cells).astype(np.int32)
    dU = rng.standard_normal(w.U.shape)
    lam = rng.standard_normal(w.U.shape)
    t = S.fill_ghosts_tangent(w.mesh, dU.copy(), table, cell_bc)
    a, vbar = S.fill_ghosts_adjoint(w.mesh, lam.copy(), table, cell_bc)
    # <lam, T dU> = <T^T lam, dU>; T maps interior rows to every row, so dU's ghost rows do not enter
    ghost = w.mesh.cell_kind == L.CELL_BOUNDARY
    dU_in = np.where(ghost[:, None], 0.0, dU)
    lhs = float(np.sum(lam * np.where(ghost[:, None], t, dU_in)))
    rhs = float(np.sum(a * dU_in))
    assert abs(lhs - rhs) <= 1e-12 * (np.abs(lam).sum() * np.abs(dU).max())
    assert np.all(a[ghost] == 0.0)
    # the value adjoint: perturbing condition b's value by e moves J = <lam, fill(U)> by <vbar[b], e>
    U = w.U.copy()
    base = float(np.sum(lam * S.fill_ghosts(w.mesh, U.copy(), table, cell_bc)))
    for b in (1, 2):
        e = rng.standard_normal(w.U.shape[1])
        tb = [list(x) for x in table]
        tb[b][1] = list(np.asarray(table[b][1]) + e)
        moved = float(np.sum(lam * S.fill_ghosts(w.mesh, U.copy(), [tuple(x) for x in tb], cell_bc)))
        assert abs((moved - base) - float(np.dot(vbar[b], e))) <= 1e-9 * (abs(base) + 1.0)


def test_pressure_gradient_matches_central_differences():
    w = workloads.wall3d(6)
    phys, keep = w.physics()
    cells, wts = w.functional
    J, G = S.pressure_functional(w.mesh, phys, w.U, cells, wts, gamma=1.4)
    assert J > 0 and G is not None
    rng = np.random.default_rng(4)
    d = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)
    eps = 1e-6
    Jp = S.pressure_functional(w.mesh, phys, w.U + eps * d, cells, wts)[0]
    Jm = S.pressure_functional(w.mesh, phys, w.U - eps * d, cells, wts)[0]
    fd = (Jp - Jm) / (2 * eps)
    assert abs(fd - float(np.sum(G * d))) <= 1e-7 * abs(fd)


def test_wall_workload_layout():
    w = workloads.wall3d(8)
    table, cell_bc = w.boundary
    g = np.nonzero(w.mesh.cell_kind == L.CELL_BOUNDARY)[0]
    x, y = w.mesh.cell_centroid[g, 0], w.mesh.cell_centroid[g, 1]
    assert np.all(cell_bc[g][x < 0] == 0) and np.all(cell_bc[g][x > 1] == 1)
    assert np.all(cell_bc[g][(y < 0) | (y > 1)] == 2)
    cells, wts = w.functional
    assert cells.size == 2 * 8 and np.unique(cells).size == cells.size
    assert np.all(w.mesh.cell_centroid[cells, 1] < 1.0 / 8) and np.all(w.mesh.cell_centroid[cells, 0] < 0.25)
    assert np.isclose(wts.sum(), 0.25)  # a quarter of the unit-length wall, unit depth
