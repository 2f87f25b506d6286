"""The oracle against the reference's RHS convergence test (compressibleFlowMmsSourceTests.cpp): for
each 2D parameter set (inviscid, with conduction, with conduction and viscosity), the residual
RHS(U_exact) + S over the central third of the unit square converges at the reference's expected L2 and
Linf orders within its tolerance of 0.2. This pins the first-order and least-squares RHS, the flux
calculators, the default (sin) limiter and the conduction and viscous fluxes against an analytic
solution."""
import numpy as np
import pytest

from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import mms


@pytest.mark.parametrize("case", mms.CASES + mms.VISCOUS_CASES, ids=[c[0] for c in mms.CASES + mms.VISCOUS_CASES])
def test_oracle_rhs_converges_at_the_reference_orders(case):
    hs, l2, li = [], [], []
    for level in range(mms.levels(case)):
        w, S, h = mms.workload(case, level)
        phys, keep = w.physics()
        F, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
        a, b = mms.residual_norms(w.mesh, F, S)
        hs.append(h)
        l2.append(a)
        li.append(b)
    s2, si = mms.slopes(hs, l2), mms.slopes(hs, li)
    np.testing.assert_allclose(s2, case[-2], atol=0.2, err_msg=f"L2 orders {s2}")
    np.testing.assert_allclose(si, case[-1], atol=0.2, err_msg=f"Linf orders {si}")


@pytest.mark.parametrize("case", [c for c in mms.VISCOUS_CASES if c[3] > 0], ids=[c[0] for c in mms.VISCOUS_CASES if c[3] > 0])
def test_viscous_sets_fail_without_the_diffusive_source(case):
    """The viscous sets test the stress and conduction terms: with the Euler source alone the momentum
    residual stops converging (orders far below the expected ones)."""
    hs, l2 = [], []
    for level in range(mms.levels(case)):
        w, _, h = mms.workload(case, level)
        X = tuple(w.mesh.cell_centroid[:, a] for a in range(w.mesh.dim))
        phys, keep = w.physics()
        F, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
        hs.append(h)
        l2.append(mms.residual_norms(w.mesh, F, mms.source(case[1], X))[0])
    s2 = mms.slopes(hs, l2)
    assert np.all(s2[2:] < np.asarray(case[-2][2:]) - 1.0), s2
