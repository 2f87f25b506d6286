"""The fused one-pass RHS (k_fused_rhs) against the two-pass kernels and the oracle.

With ABL_FV_FUSED=1 at create, where a tile's staged rows fit in shared memory, the handle runs the
fused kernel; otherwise (the default) the gradient pass + tile flux pass. Both evaluate every gradient and face flux with the
same arithmetic; they differ only in the order a cell sums its face fluxes (the fused kernel sums
opposite faces next to each other), so they agree to rounding. Both match the oracle at the FP64 bar.
"""
import os

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu

FUSED_CASES = ["tgv3d_ausmpup_lsq_minmod_visc", "tgv3d_natural_order", "sod2d_ausm_upwind", "box1d_visc", "box1d_visc_periodic",
               "box2d_ausm_minmod_const", "box2d_ausmpup_vanleer_suth", "box2d_riemann_vanalbada_none", "box2d_avg_sin_const",
               "box2d_off_zero_const", "tets3d_pg_minmod", "pgspecies3d_ns2", "walled_channel3d"]


def _solver(w, fused: bool):
    old = os.environ.get("ABL_FV_FUSED")
    os.environ["ABL_FV_FUSED"] = "1" if fused else "0"
    try:
        s = w.solver()
    finally:
        if old is None:
            del os.environ["ABL_FV_FUSED"]
        else:
            os.environ["ABL_FV_FUSED"] = old
    s.SetAux(initial_aux(w))
    return s


def _rhs(s, U, precision):
    F = np.zeros_like(U)
    s.ComputeRHSFunction(0.0, U, F, precision)
    assert s.Status() == L.OK
    return F


@pytest.mark.parametrize("name", FUSED_CASES)
def test_fused_matches_two_pass_and_oracle(name):
    w = R.case(name)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    fused, two = _solver(w, True), _solver(w, False)
    assert fused.FusedInfo()["fp64"], f"{name}: the fused kernel should fit this case"
    assert not two.FusedInfo()["fp64"]
    phys, keep = w.physics()
    F_ref, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    precisions = [L.PRECISION_FP64] + ([L.PRECISION_MIXED] if fused.FusedInfo()["mixed"] else [])
    for prec in precisions:
        Ff = _rhs(fused, w.U, prec)
        Ft = _rhs(two, w.U, prec)
        assert np.all(Ff[~owned] == 0.0)
        for block, e in R.block_errors(Ff, Ft, owned, 2 + w.mesh.dim).items():
            # the walled channel's residual is a small difference of large face fluxes: a different
            # summation order moves it by ~1e-14 of itself
            assert e <= 1e-13, f"{name} precision {prec} {block}: fused vs two-pass {e:.3e}"
        if prec == L.PRECISION_FP64:
            for block, e in R.block_errors(Ff, F_ref, owned, 2 + w.mesh.dim).items():
                assert e <= 1e-12, f"{name} {block}: fused vs oracle {e:.3e}"
    fused.close()
    two.close()


def test_fused_uniform_state_has_an_exactly_zero_residual():
    # opposite faces are summed next to each other, so equal and opposite fluxes cancel exactly
    w = R.case("tgv3d_ausmpup_lsq_minmod_visc")
    U = np.tile(np.array([1.17, 2.6e5, 40.0, -25.0, 12.5]), (w.mesh.n_cells, 1))
    s = _solver(w, True)
    for prec in (L.PRECISION_FP64, L.PRECISION_MIXED):
        F = _rhs(s, U, prec)
        assert np.all(F == 0.0), (prec, np.abs(F).max())
    s.close()


def test_fused_large_box_matches_two_pass():
    # a power-of-two box: every Morton run of 256 cells is an 8x8x4 block, one table class; and a 48^3
    # box, whose runs are not aligned blocks (many classes); FP64 and mixed
    from ablate_b200 import workloads
    w = workloads.tgv3d(32)
    fused = _solver(w, True)
    assert fused.FusedInfo()["tile_classes"] == 1 and fused.FusedInfo()["max_staged_cells"] == 848
    fused.close()
    w = workloads.tgv3d(48)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    fused, two = _solver(w, True), _solver(w, False)
    for prec in (L.PRECISION_FP64, L.PRECISION_MIXED):
        for block, e in R.block_errors(_rhs(fused, w.U, prec), _rhs(two, w.U, prec), owned, 5).items():
            assert e <= 1e-14, (prec, block, e)
    fused.close()
    two.close()
