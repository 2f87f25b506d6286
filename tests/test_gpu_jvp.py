"""Forward tangent (JVP) of the RHS through the C ABI (abl_fv_jvp_host).

Checked against
* central finite differences of the device RHS (eps 1e-7 relative to the state);
* the finite-difference Jacobian-vector product PETSc's MatMFFD would form on the reference RHS
  (Walker-Pernice step h = sqrt(eps_machine) sqrt(1 + |u|) / |a|, one-sided), evaluated on the oracle;
* linearity in the direction, and F returned alongside equal to the RHS.

The finite-difference checks run at a generic point: the seeded states are moved by 0.1% seeded noise
first. The Taylor-Green state is symmetric, so neighbouring limiter ratios tie exactly and the RHS has a
kink right at that state (forward and backward differences of the oracle differ by 1.7% there, at any
step); the tangent is then the derivative of the branch the primal takes, which no difference quotient
reproduces.
"""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu

CASES = ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausm_upwind_none", "box2d_ausmpup_vanleer_suth", "box2d_riemann_vanalbada_none",
         "species3d_ns5", "species3d_ns5_dk", "compact3d_avg_ns5", "box1d_visc", "box1d_visc_periodic", "pgspecies3d_ns2", "sod2d_ausm_upwind", "tets3d_ns9", "tets3d_pg_minmod"]


def _direction(w, seed):
    rng = np.random.default_rng(seed)
    scale = np.abs(w.U).mean(0)
    scale = np.where(scale > 0, scale, 1e-2 * np.sqrt(scale[0] * scale[1]))  # momentum of a fluid at rest
    dU = rng.standard_normal(w.U.shape) * scale * 1e-2
    dU[w.mesh.cell_kind == L.CELL_BOUNDARY] = 0.0  # boundary ghost values are not unknowns of the RHS
    return dU


def _generic(w):
    # 0.1% relative noise; vanishing components (the momentum of a fluid at rest) get absolute noise,
    # which moves the state off the u = 0 switch of the upwind direction
    rng = np.random.default_rng(11)
    U = w.U * (1.0 + 1e-3 * rng.standard_normal(w.U.shape))
    s = np.abs(w.U).mean(0)
    zero = s == 0
    U[:, zero] += 1e-5 * np.sqrt(s[0] * s[1]) * rng.standard_normal((w.U.shape[0], int(zero.sum())))
    return np.ascontiguousarray(U)


def _rhs(s, w, U):
    F = np.zeros_like(U)
    s.ComputeRHSFunction(0.0, U, F)
    return F


def _rel(a, b, owned):
    return np.linalg.norm(a[owned] - b[owned]) / np.linalg.norm(b[owned])


@pytest.mark.parametrize("name", CASES)
def test_jvp_matches_central_differences(name):
    w = R.case(name)
    s = w.solver()
    s.SetAux(initial_aux(w))
    U = _generic(w)
    dU = _direction(w, 1)
    dF = np.zeros_like(w.U)
    F = np.zeros_like(w.U)
    s.ComputeJVP(0.0, U, dU, dF, F)
    assert s.Status() == L.OK
    owned = w.mesh.cell_kind == L.CELL_OWNED
    eps = 1e-7 / 1e-2  # dU is ~1e-2 of the state: 1e-7 relative perturbation
    Fp = _rhs(s, w, U + eps * dU)
    Fm = _rhs(s, w, U - eps * dU)
    fd = (Fp - Fm) / (2 * eps)
    assert _rel(dF, fd, owned) < 2e-5, _rel(dF, fd, owned)
    # the value returned with the tangent is the RHS
    F0 = _rhs(s, w, U)
    assert _rel(F, F0, owned) < 1e-12


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausm_upwind_none", "species3d_ns5"])
def test_jvp_matches_petsc_style_fd_of_the_oracle(name):
    w = R.case(name)
    phys, keep = w.physics()
    s = w.solver()
    s.SetAux(initial_aux(w))
    U = _generic(w)
    dU = _direction(w, 2)
    dF = np.zeros_like(w.U)
    s.ComputeJVP(0.0, U, dU, dF)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    # MatMFFD "wp" differencing parameter: h = error_rel * sqrt(1 + ||u||) / ||a||, error_rel = sqrt(eps)
    h = np.sqrt(np.finfo(float).eps) * np.sqrt(1.0 + np.linalg.norm(U[owned])) / np.linalg.norm(dU[owned])
    F0, _ = orc.rhs(w.mesh, phys, U, initial_aux(w))
    F1, _ = orc.rhs(w.mesh, phys, U + h * dU, initial_aux(w))
    fd = (F1 - F0) / h
    # With the NASA-7 mixture the reference's temperature secant stops at |e - e(T)| <= 1e-8 J/kg, which
    # limits the one-sided quotient at this tiny step to about 1e-3 of the tangent.
    tol = 1e-3 if isinstance(w.eos, fv.TChem) else 1e-4
    assert _rel(dF, fd, owned) < tol, _rel(dF, fd, owned)


def test_jvp_is_linear_in_the_direction():
    w = R.case("tgv3d_ausmpup_lsq_minmod_visc")
    s = w.solver()
    a, b = _direction(w, 3), _direction(w, 4)
    Ja, Jb, Jab = (np.zeros_like(w.U) for _ in range(3))
    s.ComputeJVP(0.0, w.U, a, Ja)
    s.ComputeJVP(0.0, w.U, b, Jb)
    s.ComputeJVP(0.0, w.U, 2.0 * a - 3.0 * b, Jab)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    assert _rel(Jab, 2.0 * Ja - 3.0 * Jb, owned) < 1e-12


def test_jvp_accumulates():
    w = R.case("box2d_ausm_minmod_const")
    s = w.solver()
    dU = _direction(w, 5)
    base = np.random.default_rng(9).standard_normal(w.U.shape)
    d1 = np.zeros_like(w.U)
    s.ComputeJVP(0.0, w.U, dU, d1)
    d2 = base.copy()
    s.ComputeJVP(0.0, w.U, dU, d2)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    np.testing.assert_allclose(d2[owned], base[owned] + d1[owned], rtol=1e-12, atol=1e-9)
    np.testing.assert_array_equal(d2[~owned], base[~owned])
