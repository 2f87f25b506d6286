"""The 1D face interpolant (faceInterpolant.cpp:32-36): in 1D the reference builds each face's stencil
with stencil::LeastSquares (src/finiteVolume/stencils/leastSquares.cpp:5-122), over the two cells
sharing the face, not LeastSquaresAverage. On a uniform mesh its face gradient is (u_R - u_L) / h.

Conduction only (no advection, mu = 0), with T = T0 + c x^4: the energy residual of an interior cell
is then k (T_{i+1} - 2 T_i + T_{i-1}) / h^2 = k (12 c x^2 + c h^2). Averaging the two cells'
least-squares gradients instead gives k (T_{i+2} - 2 T_i + T_{i-2}) / (4 h^2) = k (12 c x^2 + 4 c h^2),
which this distinguishes.
"""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.mesh import box_mesh
from ablate_b200.workloads import Workload, initial_aux
from oracle import oracle as orc

R_GAS = 287.0


def _conduction_residual(n, periodic, T_of_x):
    mesh = box_mesh((n,), periodic=(periodic,))
    eos = fv.PerfectGas({"gamma": 1.4, "Rgas": R_GAS})
    x = mesh.cell_centroid[:, 0]
    T = T_of_x(x)
    U = np.zeros((mesh.n_cells, 3))
    U[:, 0] = 1.0
    U[:, 1] = 1.0 * R_GAS * T / 0.4  # rho e with p = rho R T, u = 0
    k = 0.7
    procs = [fv.NavierStokesTransport({}, eos, None, fv.Constant(k=k, mu=0.0))]
    w = Workload("cond1d", mesh, eos, procs, "upwind", "none", U, "1D conduction")
    phys, keep = w.physics()
    F, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    return mesh, F, T, k


@pytest.mark.parametrize("periodic", [False, True])
def test_1d_face_gradient_is_the_two_cell_difference(periodic):
    n = 24
    mesh, F, T, k = _conduction_residual(n, periodic, lambda x: 300.0 + 80.0 * x ** 4)
    h = 1.0 / n
    own = np.flatnonzero(mesh.cell_kind == L.CELL_OWNED)
    order = own[np.argsort(mesh.cell_centroid[own, 0])]
    To = T[order]
    inner = slice(1, n - 1)
    expect = k * (To[2:] - 2 * To[1:-1] + To[:-2]) / h ** 2
    got = F[order, 1][inner]
    np.testing.assert_allclose(got, expect, rtol=1e-9, atol=1e-9 * np.abs(expect).max())


def test_averaged_gradients_would_differ():
    # the residual from averaged cell gradients (the 2D/3D LeastSquaresAverage form) is off by
    # 3 k c h^2; make sure the check above can see that size
    n, c, k = 24, 80.0, 0.7
    h = 1.0 / n
    x = (np.arange(n) + 0.5) * h
    T = 300.0 + c * x ** 4
    two_point = k * (T[2:] - 2 * T[1:-1] + T[:-2]) / h ** 2
    g = np.gradient(T, h)  # central differences in the interior
    gf = 0.5 * (g[1:] + g[:-1])
    averaged = k * (gf[1:] - gf[:-1]) / h
    assert np.abs(averaged[1:-1] - two_point[1:-1]).max() > 1e-6 * np.abs(two_point).max()
