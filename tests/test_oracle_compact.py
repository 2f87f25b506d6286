"""CompactCompressibleNSSpeciesTransport (src/finiteVolume/processes/compactCompressibleNSSpeciesTransport.cpp)
on the oracle. Its fluxes are NavierStokesTransport's and SpeciesTransport's, except the species
advection where the flux calculator gives no direction (NA, e.g. AverageFlux): there rho Y_k is carried
as (rho Y_L + rho Y_R) / (rho_L + rho_R) (:257-259) where SpeciesTransport takes the right state
(speciesTransport.cpp:330-338).
"""
import numpy as np
import pytest

from ablate_b200 import fv
from ablate_b200.workloads import Workload, initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R


def _workload(flux, compact):
    w0 = R.case("species3d_ns5")
    tr = fv.Constant(k=0.03, mu=2e-5, diff=5e-5)
    if compact:
        procs = [fv.CompactCompressibleNSSpeciesTransport({}, w0.eos, flux, tr)]
    else:
        procs = [fv.NavierStokesTransport({}, w0.eos, flux, tr), fv.SpeciesTransport(w0.eos, flux, tr)]
    return Workload(w0.name, w0.mesh, w0.eos, procs, w0.petscfv_type, w0.limiter, w0.U, w0.description)


def _rhs(w):
    phys, keep = w.physics()
    return orc.rhs(w.mesh, phys, w.U, initial_aux(w))[0]


@pytest.mark.parametrize("compact", [False, True])
def test_face_flux_without_direction(compact):
    w = _workload(fv.AverageFlux(), compact)
    phys, keep = w.physics()
    rng = np.random.default_rng(3)
    ne = 5
    for _ in range(5):
        a, b = w.U[rng.integers(len(w.U))], w.U[rng.integers(len(w.U))]
        normal = rng.standard_normal(3) * 0.01
        mA = orc.ns_advection_flux(phys, 3, normal, a[:ne], b[:ne], 600.0, 650.0)[0]
        fs = orc.species_advection_flux(phys, 3, normal, a, b, 600.0, 650.0)
        expect = mA * (a[ne:] + b[ne:]) / (a[0] + b[0]) if compact else mA * b[ne:] / b[0]
        np.testing.assert_allclose(fs, expect, rtol=1e-13, atol=1e-13 * np.abs(expect).max())


def test_compact_equals_the_two_processes_when_the_flux_has_a_direction():
    assert np.array_equal(_rhs(_workload(fv.Ausm(), True)), _rhs(_workload(fv.Ausm(), False)))


def test_compact_average_flux_differs_only_in_the_species():
    Fc, Fs = _rhs(_workload(fv.AverageFlux(), True)), _rhs(_workload(fv.AverageFlux(), False))
    assert np.array_equal(Fc[:, :5], Fs[:, :5])
    assert not np.allclose(Fc[:, 5:], Fs[:, 5:], rtol=1e-6, atol=0)
