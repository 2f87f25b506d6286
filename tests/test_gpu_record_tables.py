"""Repeated geometry and weight records stored once (abl_fv_record_classes).

On structured blocks every tile face of one orientation has the same geometry record and every
interior cell the same cone weights; the device then stores each distinct record once and reads it
through a per-face / per-cell index. The arithmetic is unchanged, so the RHS (FP64 and mixed), the JVP
and the VJP must equal, bit for bit, those of the one-record-per-face layout (ABL_FV_RECORD_TABLES=0).
Unstructured meshes keep one record per face and cone entry.
"""
import os

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import workloads
from ablate_b200.workloads import initial_aux
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu


def _workload(name):
    if name == "tgv3d_16":
        return workloads.tgv3d(16)
    if name.startswith("wall3d_"):
        return workloads.wall3d(int(name.split("_")[1]))
    return R.case(name)


def _solver(w, tables: bool):
    old = os.environ.get("ABL_FV_RECORD_TABLES")
    os.environ["ABL_FV_RECORD_TABLES"] = "1" if tables else "0"
    try:
        s = w.solver()
    finally:
        if old is None:
            del os.environ["ABL_FV_RECORD_TABLES"]
        else:
            os.environ["ABL_FV_RECORD_TABLES"] = old
    s.SetAux(initial_aux(w))
    return s


def _outputs(s, w):
    rng = np.random.default_rng(5)
    U = w.U * (1.0 + 1e-3 * rng.standard_normal(w.U.shape))
    dU = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)
    Fbar = rng.standard_normal(w.U.shape)
    out = {}
    F = np.zeros_like(U)
    s.ComputeRHSFunction(0.0, U, F, L.PRECISION_FP64)
    out["rhs"] = F
    if s.nc == s.mesh.dim + 2:
        Fm = np.zeros_like(U)
        s.ComputeRHSFunction(0.0, U, Fm, L.PRECISION_MIXED)
        out["mixed"] = Fm
    dF, Fj = np.zeros_like(U), np.zeros_like(U)
    s.ComputeJVP(0.0, U, dU, dF, Fj)
    out["jvp"] = dF
    Ub = np.zeros_like(U)
    s.ComputeVJP(0.0, U, Fbar, Ub)
    out["vjp"] = Ub
    assert s.Status() == L.OK
    return out


# wall3d_12: spacing 1/12 is not exact in binary, so the cone weights differ in their last bits from
# cell to cell and only the geometry records repeat (weight tables off, geometry table on)
NAMES = ["tgv3d_16", "wall3d_16", "wall3d_12"] + R.CASES


@pytest.mark.parametrize("name", NAMES)
def test_record_tables_give_bitwise_the_same_results(name):
    w = _workload(name)
    a = _solver(w, True)
    b = _solver(w, False)
    try:
        assert b.RecordClasses() == (0, 0)
        ra, rb = _outputs(a, w), _outputs(b, w)
        for key in ra:
            assert np.array_equal(ra[key], rb[key]), f"{key} differs between the layouts ({a.RecordClasses()})"
    finally:
        a.close()
        b.close()


def test_structured_blocks_use_tables_and_unstructured_meshes_do_not():
    for name, structured in [("tgv3d_16", True), ("wall3d_16", True), ("sod2d_ausm_upwind", True), ("tets3d_ns9", False)]:
        w = _workload(name)
        s = _solver(w, True)
        try:
            wc, gc = s.RecordClasses()
        finally:
            s.close()
        if structured:
            assert 0 < gc <= 64, (name, wc, gc)
            assert 0 < wc <= 64 or name == "sod2d_ausm_upwind", (name, wc, gc)
        else:
            assert (wc, gc) == (0, 0), (name, wc, gc)
