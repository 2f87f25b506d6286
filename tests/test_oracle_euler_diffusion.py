"""The oracle against the reference's 1D conduction convergence test
(compressibleFlowEulerDiffusionTests.cpp): order 2.25 for rho E (L2 and Linf, within 0.2), rho and
rho u exact. In 1D the face gradient comes from the two-cell LeastSquares stencil, so this pins it."""
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import euler_diffusion as ED


def test_oracle_conduction_converges_at_the_reference_order():
    hs, l2, li = [], [], []
    for level in range(ED.LEVELS):
        w, h = ED.workload(level)
        phys, keep = w.physics()
        aux = initial_aux(w)
        U, t = ED.march(w, lambda U: orc.rhs(w.mesh, phys, U, aux)[0])
        a, b = ED.errors(w, U, t)
        assert a[0] == 0.0 and a[2] == 0.0 and b[0] == 0.0 and b[2] == 0.0, (a, b)
        hs.append(h)
        l2.append(a[1])
        li.append(b[1])
    s2, si = ED.slope(hs, l2), ED.slope(hs, li)
    assert abs(s2 - ED.EXPECTED) <= 0.2, s2
    assert abs(si - ED.EXPECTED) <= 0.2, si
