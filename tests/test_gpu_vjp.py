"""Adjoint (VJP) of the RHS through the C ABI (abl_fv_vjp_host).

Checked against
* the tangent: <w, J v> from abl_fv_jvp equals <J^T w, v> from abl_fv_vjp for seeded w, v (the
  dot-product test of an adjoint), over every cell including boundary ghosts;
* central finite differences of the scalar <w, F(U)> along v, F from the device RHS;
* PETSc-style one-sided differences of the same scalar on the oracle RHS;
* accumulation (Ubar += ...) and linearity in w.

Like the tangent tests, these run at a generic point (the seeded state moved by 0.1% seeded noise), away
from the kinks of the limiter minimum on the symmetric Taylor-Green state.
"""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu

CASES = ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausm_upwind_none", "box2d_ausm_minmod_const", "box2d_ausmpup_vanleer_suth",
         "box2d_riemann_vanalbada_none", "box2d_avg_sin_const", "box2d_off_zero_const", "box1d_riemann_upwind", "sod2d_ausm_upwind",
         "species3d_ns5", "species3d_ns9", "species3d_ns5_dk", "compact3d_avg_ns5", "box1d_visc", "box1d_visc_periodic", "pgspecies3d_ns2", "tets3d_ns9", "tets3d_pg_minmod"]


def _scale(U):
    # typical magnitude per component; a component that vanishes in the state (the momentum of a fluid
    # at rest) takes a velocity of a few m/s
    s = np.abs(U).mean(0)
    return np.where(s > 0, s, 1e-2 * np.sqrt(s[0] * s[1]))


def _generic(w):
    # 0.1% relative noise; vanishing components get absolute noise on the same scale, which moves a
    # fluid at rest off the u = 0 switch of the upwind direction
    rng = np.random.default_rng(11)
    U = w.U * (1.0 + 1e-3 * rng.standard_normal(w.U.shape))
    zero = np.abs(w.U).mean(0) == 0
    U[:, zero] += 1e-3 * _scale(w.U)[zero] * rng.standard_normal((w.U.shape[0], int(zero.sum())))
    return np.ascontiguousarray(U)


def _vectors(w, seed):
    rng = np.random.default_rng(seed)
    scale = _scale(w.U)
    v = rng.standard_normal(w.U.shape) * scale * 1e-2
    wt = rng.standard_normal(w.U.shape) / scale
    wt[w.mesh.cell_kind != L.CELL_OWNED] = 0.0  # the RHS has rows on owned cells only
    return np.ascontiguousarray(v), np.ascontiguousarray(wt)


def _vjp(s, U, wt):
    Ub = np.zeros_like(U)
    s.ComputeVJP(0.0, U, wt, Ub)
    assert s.Status() == L.OK
    return Ub


def _jvp(s, U, v):
    dF = np.zeros_like(U)
    s.ComputeJVP(0.0, U, v, dF)
    return dF


@pytest.mark.parametrize("name", CASES)
def test_vjp_is_the_transpose_of_the_jvp(name):
    w = R.case(name)
    s = w.solver()
    s.SetAux(initial_aux(w))
    U = _generic(w)
    for seed in (1, 2):
        v, wt = _vectors(w, seed)
        Jv = _jvp(s, U, v)
        lhs = float(np.sum(wt * Jv))
        rhs = float(np.sum(_vjp(s, U, wt) * v))
        # both sides are sums of ~1e3 terms of either sign: bound by the terms' magnitude
        assert abs(lhs - rhs) <= 1e-12 * float(np.sum(np.abs(wt * Jv))), (lhs, rhs)


@pytest.mark.parametrize("name", CASES)
def test_vjp_matches_central_differences(name):
    w = R.case(name)
    s = w.solver()
    s.SetAux(initial_aux(w))
    U = _generic(w)
    v, wt = _vectors(w, 3)
    g = float(np.sum(_vjp(s, U, wt) * v))

    eps = 1e-7 / 1e-2
    Fp, Fm = np.zeros_like(U), np.zeros_like(U)
    s.ComputeRHSFunction(0.0, U + eps * v, Fp)
    s.ComputeRHSFunction(0.0, U - eps * v, Fm)
    fdv = (Fp - Fm) / (2 * eps)
    fd = float(np.sum(wt * fdv))
    # the error bound of the difference quotient, projected: 2e-5 of ||w o fd||_1
    assert abs(g - fd) <= 2e-5 * float(np.sum(np.abs(wt * fdv))), (g, fd)


@pytest.mark.parametrize("name", ["tgv3d_ausmpup_lsq_minmod_visc", "box2d_ausmpup_vanleer_suth", "species3d_ns5"])
def test_vjp_matches_petsc_style_fd_of_the_oracle(name):
    w = R.case(name)
    phys, keep = w.physics()
    s = w.solver()
    s.SetAux(initial_aux(w))
    U = _generic(w)
    v, wt = _vectors(w, 4)
    v[w.mesh.cell_kind == L.CELL_BOUNDARY] = 0.0
    g = float(np.sum(_vjp(s, U, wt) * v))
    owned = w.mesh.cell_kind == L.CELL_OWNED
    h = np.sqrt(np.finfo(float).eps) * np.sqrt(1.0 + np.linalg.norm(U[owned])) / np.linalg.norm(v[owned])
    F0, _ = orc.rhs(w.mesh, phys, U, initial_aux(w))
    F1, _ = orc.rhs(w.mesh, phys, U + h * v, initial_aux(w))
    fdv = (F1 - F0) / h
    fd = float(np.sum(wt * fdv))
    tol = 1e-3 if isinstance(w.eos, fv.TChem) else 1e-4
    assert abs(g - fd) <= tol * float(np.sum(np.abs(wt * fdv))), (g, fd)


def test_vjp_accumulates_and_is_linear():
    w = R.case("tgv3d_ausmpup_lsq_minmod_visc")
    s = w.solver()
    U = _generic(w)
    _, a = _vectors(w, 5)
    _, b = _vectors(w, 6)
    Ja, Jb = _vjp(s, U, a), _vjp(s, U, b)
    base = np.random.default_rng(9).standard_normal(U.shape)
    acc = base.copy()
    s.ComputeVJP(0.0, U, 2.0 * a - 3.0 * b, acc)
    ref = base + 2.0 * Ja - 3.0 * Jb
    assert np.linalg.norm(acc - ref) <= 1e-12 * np.linalg.norm(ref)
