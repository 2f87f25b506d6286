"""The oracle against the reference's species advection convergence test
(compressibleFlowSpeciesAdvectionTests.cpp): first-order species advection converges at order 1
(L2 and Linf, within 0.2) and the uniform Euler state is kept exactly."""
import numpy as np

from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import species_advection as SA


def test_oracle_species_advection_converges_at_order_one():
    hs, l2, li = [], [], []
    for level in range(SA.LEVELS):
        w, h = SA.workload(level)
        phys, keep = w.physics()
        aux = initial_aux(w)
        U, t = SA.march(w, lambda t, U: orc.rhs(w.mesh, phys, U, aux)[0])
        a, b = SA.errors(w, U, t)
        assert np.all(a[:4] == 0.0) and np.all(b[:4] == 0.0), (a[:4], b[:4])
        hs.append(h)
        l2.append(a[4:])
        li.append(b[4:])
    s2, si = SA.slopes(hs, l2), SA.slopes(hs, li)
    np.testing.assert_allclose(s2, SA.EXPECTED, atol=0.2, err_msg=f"L2 orders {s2}")
    np.testing.assert_allclose(si, SA.EXPECTED, atol=0.2, err_msg=f"Linf orders {si}")
