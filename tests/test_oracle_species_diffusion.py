"""The oracle against the reference's 1D species diffusion convergence test
(compressibleFlowSpeciesDiffusionTests.cpp), its four single-rank parameter sets (density 1 and 2,
the diffusivity scalar or one per species): order 2.2 for rho Y0 and rho Y1 (L2 and Linf, within
0.2); rho, rho E and rho u exact and rho Y2 to rounding. The device has no 1D species build; the
reference's rho E check needs its mock enthalpies and is not ported (tests/species_diffusion.py)."""
import numpy as np
import pytest

from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import species_diffusion as SD


@pytest.mark.parametrize("rho,vector", [(1.0, False), (2.0, False), (1.0, True), (2.0, True)])
def test_oracle_species_diffusion_converges_at_the_reference_order(rho, vector):
    hs, l2, li = [], [], []
    for level in SD.LEVELS:
        w, h = SD.workload(level, rho, vector)
        phys, keep = w.physics()
        aux = initial_aux(w)
        U, t = SD.march(w, lambda U: orc.rhs(w.mesh, phys, U, aux)[0], rho)
        a, b = SD.errors(w, U, t, rho)
        assert np.all(b[:3] == 0.0), b
        assert b[5] <= 1e-14 * rho, b
        hs.append(h)
        l2.append(a)
        li.append(b)
    l2, li = np.array(l2), np.array(li)
    for c, order in SD.EXPECTED.items():
        assert abs(SD.slope(hs, l2[:, c]) - order) <= 0.2, (c, SD.slope(hs, l2[:, c]))
        assert abs(SD.slope(hs, li[:, c]) - order) <= 0.2, (c, SD.slope(hs, li[:, c]))
