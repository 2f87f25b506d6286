"""Failure paths of the C ABI: corrupt descriptors rejected on the host, and the device status word's
EOS iteration cap.

The host-side checks need no GPU: abl_fv_create validates the physics and sets the mesh up on the host
before it looks for a device, so every rejection below has the same code with or without one. The EOS
case runs the mixture temperature's secant iteration to its cap (two passes of at most 100 steps, a
bounded loop) and reads the status word; nothing in this file faults or hangs a device.
"""
import ctypes as C

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.mesh import box_mesh
from tests import golden_cases as G


def _gas(ns=0):
    p = L.PhysicsDesc()
    p.eos, p.gamma, p.r_gas, p.flux, p.advection, p.n_species = L.EOS_PERFECT_GAS, 1.4, 287.0, L.FLUX_AUSM, 1, ns
    return p


def _create(mesh_desc, phys):
    h = C.c_void_p()
    rc = L.lib.abl_fv_create(C.byref(mesh_desc), C.byref(phys), 0, C.byref(h))
    if h.value:
        L.lib.abl_fv_destroy(h)
    return rc, L.lib.abl_last_error_string()


def test_species_count_above_the_cap_is_rejected():
    m = box_mesh((4, 4))
    d = m.desc()
    rc, msg = _create(d, _gas(ns=129))
    assert rc == L.ERR_INVALID_ARGUMENT and b"n_species out of range" in msg
    z = np.zeros(8)
    assert L.lib.abl_eos_batch(C.byref(_gas(ns=129)), 3, L.PROP_PRESSURE, 1, L.dptr(z), None, L.dptr(z)) == L.ERR_INVALID_ARGUMENT
    rc, msg = _create(d, _gas(ns=-1))
    assert rc == L.ERR_INVALID_ARGUMENT


def _corrupt(edit):
    """A 4x3 box (outflow ghosts on x, periodic in y) with one edit applied to its arrays."""
    m = box_mesh((4, 3), periodic=(False, True))
    arrays = {"face_cells": m.face_cells.copy(), "cell_volume": m.cell_volume.copy(), "cell_kind": m.cell_kind.copy()}
    edit(m, arrays)
    m.face_cells, m.cell_volume, m.cell_kind = arrays["face_cells"], arrays["cell_volume"], arrays["cell_kind"]
    return m.desc()


def _interior_face(m):
    k = m.cell_kind
    return int(np.nonzero((k[m.face_cells[:, 0]] == L.CELL_OWNED) & (k[m.face_cells[:, 1]] == L.CELL_OWNED))[0][0])


@pytest.mark.parametrize("what,edit,needle", [
    ("support out of range", lambda m, a: a["face_cells"].__setitem__((0, 1), m.n_cells), b"invalid support"),
    ("negative support", lambda m, a: a["face_cells"].__setitem__((0, 0), -1), b"invalid support"),
    ("face with one cell on both sides", lambda m, a: a["face_cells"].__setitem__((0, 1), a["face_cells"][0, 0]), b"invalid support"),
    ("zero volume", lambda m, a: a["cell_volume"].__setitem__(2, 0.0), b"volume must be positive"),
    ("negative volume", lambda m, a: a["cell_volume"].__setitem__(5, -1e-3), b"volume must be positive"),
    ("NaN volume", lambda m, a: a["cell_volume"].__setitem__(1, np.nan), b"volume must be positive"),
    ("unknown cell kind", lambda m, a: a["cell_kind"].__setitem__(0, 9), b"invalid cell kind"),
    # an interior cell relabelled as a boundary ghost has four faces: a ghost must have exactly one
    ("ghost with several faces", lambda m, a: a["cell_kind"].__setitem__(int(m.face_cells[_interior_face(m), 0]), L.CELL_BOUNDARY),
     b"exactly one face"),
])
def test_corrupt_mesh_descriptor_is_rejected(what, edit, needle):
    d = _corrupt(edit)
    rc, msg = _create(d, _gas())
    assert rc == L.ERR_INVALID_ARGUMENT, (what, rc, msg)
    assert needle in msg, (what, msg)


def test_empty_mesh_descriptor_is_rejected():
    d = box_mesh((3, 3)).desc()
    d.n_cells = 0
    rc, msg = _create(d, _gas())
    assert rc == L.ERR_INVALID_ARGUMENT and b"invalid mesh descriptor" in msg
    d = box_mesh((3, 3)).desc()
    d.dim = 4
    assert _create(d, _gas())[0] == L.ERR_INVALID_ARGUMENT


# ---- device status word ---------------------------------------------------------------------------
def _below_one_kelvin(eos, U, rows, dim):
    """Set the internal energy of `rows` far below the mixture's e_s(1 K): the secant iteration clamps T at
    1 K and runs out of steps (TChem's Temperature_TemplateRun returns its last iterate silently; the
    device raises the status bit instead)."""
    U = U.copy()
    rho = U[rows, 0]
    ke = 0.5 * (U[rows, 2:2 + dim] ** 2).sum(1) / rho
    U[rows, 1] = rho * (-1e9) + ke
    return U


@pytest.mark.gpu
def test_eos_iteration_cap_reported_by_the_batch():
    c, phys, keep, dim, u = next(iter(G.tchem_cases()))
    U = np.ascontiguousarray(np.repeat(u, 4, axis=0))
    bad = _below_one_kelvin(None, U, [2], dim)
    out = np.zeros((4, 1))
    rc = L.lib.abl_eos_batch(C.byref(phys), dim, L.PROP_TEMPERATURE, 4, L.dptr(bad), None, L.dptr(out))
    assert rc == L.ERR_EOS_NOT_CONVERGED
    assert b"did not converge" in L.lib.abl_last_error_string()
    # the good rows are unaffected by the failing one
    rc = L.lib.abl_eos_batch(C.byref(phys), dim, L.PROP_TEMPERATURE, 4, L.dptr(U), None, L.dptr(out))
    assert rc == L.OK


@pytest.mark.gpu
def test_eos_iteration_cap_reported_by_the_rhs_status():
    from tests import rhs_cases as R
    from ablate_b200.workloads import initial_aux
    w = R.case("species3d_ns5")
    owned = np.nonzero(w.mesh.cell_kind == L.CELL_OWNED)[0]
    U = _below_one_kelvin(w.eos, w.U, [int(owned[7])], w.mesh.dim)
    s = w.solver()
    s.SetAux(initial_aux(w))
    F = np.zeros_like(U)
    s.ComputeRHSFunction(0.0, U, F, L.PRECISION_FP64)
    assert s.Status() == L.ERR_EOS_NOT_CONVERGED
    assert s.Status() == L.OK  # reading clears the word
    s.close()
