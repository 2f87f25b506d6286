"""The device RHS on the reference's species advection convergence test
(compressibleFlowSpeciesAdvectionTests.cpp; 2D, three species in a perfect gas): order 1 for the
species, the Euler state kept exactly, and after the 50 steps of every level the device state equals
the oracle's to 1e-12 of its norm."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import species_advection as SA

pytestmark = pytest.mark.gpu


def test_device_species_advection_converges_at_order_one():
    hs, l2, li = [], [], []
    for level in range(SA.LEVELS):
        w, h = SA.workload(level)
        s = w.solver()
        aux = initial_aux(w)
        s.SetAux(aux)

        def rhs(t, U):
            F = np.zeros_like(U)
            s.ComputeRHSFunction(t, U, F, L.PRECISION_FP64)
            return F

        U, t = SA.march(w, rhs)
        assert s.Status() == L.OK
        s.close()
        phys, keep = w.physics()
        U_ref, _ = SA.march(w, lambda t, U: orc.rhs(w.mesh, phys, U, aux)[0])
        own = w.mesh.cell_kind == L.CELL_OWNED
        assert np.linalg.norm(U[own] - U_ref[own]) <= 1e-12 * np.linalg.norm(U_ref[own])
        a, b = SA.errors(w, U, t)
        assert np.all(a[:4] == 0.0) and np.all(b[:4] == 0.0), (a[:4], b[:4])
        hs.append(h)
        l2.append(a[4:])
        li.append(b[4:])
    s2, si = SA.slopes(hs, l2), SA.slopes(hs, li)
    np.testing.assert_allclose(s2, SA.EXPECTED, atol=0.2, err_msg=f"L2 orders {s2}")
    np.testing.assert_allclose(si, SA.EXPECTED, atol=0.2, err_msg=f"Linf orders {si}")
