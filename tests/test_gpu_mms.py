"""The device RHS against the reference's RHS convergence test (compressibleFlowMmsSourceTests.cpp):
the same convergence orders as the reference expects, and at every level the device residual equals
the oracle's to 1e-12 of its norm."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import mms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", mms.CASES + mms.VISCOUS_CASES, ids=[c[0] for c in mms.CASES + mms.VISCOUS_CASES])
def test_device_rhs_converges_at_the_reference_orders(case):
    hs, l2, li = [], [], []
    for level in range(mms.levels(case)):
        w, S, h = mms.workload(case, level)
        s = w.solver()
        s.SetAux(initial_aux(w))
        F = np.zeros_like(w.U)
        s.ComputeRHSFunction(0.0, w.U, F, L.PRECISION_FP64)
        assert s.Status() == L.OK
        s.close()
        phys, keep = w.physics()
        F_ref, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
        owned = w.mesh.cell_kind == L.CELL_OWNED
        assert np.linalg.norm(F[owned] - F_ref[owned]) <= 1e-12 * np.linalg.norm(F_ref[owned])
        a, b = mms.residual_norms(w.mesh, F, S)
        hs.append(h)
        l2.append(a)
        li.append(b)
    s2, si = mms.slopes(hs, l2), mms.slopes(hs, li)
    np.testing.assert_allclose(s2, case[-2], atol=0.2, err_msg=f"L2 orders {s2}")
    np.testing.assert_allclose(si, case[-1], atol=0.2, err_msg=f"Linf orders {si}")
