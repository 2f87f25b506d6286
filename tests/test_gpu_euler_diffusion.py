"""The device RHS on the reference's 1D conduction convergence test
(compressibleFlowEulerDiffusionTests.cpp): order 2.25 for rho E within 0.2, rho and rho u exact,
and after the 600 steps of every level the device state equals the oracle's to 1e-12 of its norm."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import euler_diffusion as ED

pytestmark = pytest.mark.gpu


def test_device_conduction_converges_at_the_reference_order():
    hs, l2, li = [], [], []
    for level in range(ED.LEVELS):
        w, h = ED.workload(level)
        s = w.solver()
        aux = initial_aux(w)
        s.SetAux(aux)

        def rhs(U):
            F = np.zeros_like(U)
            s.ComputeRHSFunction(0.0, U, F, L.PRECISION_FP64)
            return F

        U, t = ED.march(w, rhs)
        assert s.Status() == L.OK
        s.close()
        phys, keep = w.physics()
        U_ref, _ = ED.march(w, lambda U: orc.rhs(w.mesh, phys, U, aux)[0])
        own = w.mesh.cell_kind == L.CELL_OWNED
        assert np.linalg.norm(U[own] - U_ref[own]) <= 1e-12 * np.linalg.norm(U_ref[own])
        a, b = ED.errors(w, U, t)
        assert a[0] == 0.0 and a[2] == 0.0 and b[0] == 0.0 and b[2] == 0.0, (a, b)
        hs.append(h)
        l2.append(a[1])
        li.append(b[1])
    s2, si = ED.slope(hs, l2), ED.slope(hs, li)
    assert abs(s2 - ED.EXPECTED) <= 0.2, s2
    assert abs(si - ED.EXPECTED) <= 0.2, si
