"""The oracle against the reference's RHS convergence test (compressibleFlowMmsSourceTests.cpp): for
each inviscid parameter set, the residual RHS(U_exact) + S over the central third of the unit square
converges at the reference's expected L2 and Linf orders within its tolerance of 0.2. This pins the
first-order and least-squares RHS, the flux calculators and the default (sin) limiter against an
analytic solution."""
import numpy as np
import pytest

from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import mms


@pytest.mark.parametrize("case", mms.CASES, ids=[c[0] for c in mms.CASES])
def test_oracle_rhs_converges_at_the_reference_orders(case):
    hs, l2, li = [], [], []
    for level in range(mms.LEVELS):
        w, S, h = mms.workload(case, level)
        phys, keep = w.physics()
        F, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
        a, b = mms.residual_norms(w.mesh, F, S)
        hs.append(h)
        l2.append(a)
        li.append(b)
    s2, si = mms.slopes(hs, l2), mms.slopes(hs, li)
    np.testing.assert_allclose(s2, case[6], atol=0.2, err_msg=f"L2 orders {s2}")
    np.testing.assert_allclose(si, case[7], atol=0.2, err_msg=f"Linf orders {si}")
