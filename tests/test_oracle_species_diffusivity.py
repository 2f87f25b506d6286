"""The oracle's species diffusion with one constant diffusivity per species (the Constant transport
model given a vector: SpeciesTransport::DiffusionSpeciesFluxVariableDiffusionCoefficient and
DiffusionEnergyFluxVariableDiffusionCoefficient, src/finiteVolume/processes/speciesTransport.cpp:154-194,
230-261). The reference selects them when the model's diffusivity has one entry per species
(speciesTransport.cpp:53-77); the species flux of species k then uses D_k where the scalar form
uses D, and the energy flux sums rho D_k h_s,k grad Y_k.

Checked without a golden file, against the scalar form the existing fixtures pin:
* every D_k equal to D gives bit for bit the scalar-D residual;
* the residual of species k with the vector equals, bit for bit, the residual of species k with the
  scalar D = D_k (its flux involves no other species' diffusivity);
* the energy residual is affine in the vector: R(D) = R(0) + sum_k (R(D_k e_k) - R(0)).
"""
import numpy as np
import pytest

from ablate_b200 import fv
from ablate_b200.workloads import Workload, initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R


def _rhs(base, diff):
    w0 = R.case(base)
    tr = fv.Constant(k=0.03, mu=2e-5, diff=diff)
    flux = fv.AusmpUp(0.3)
    procs = [fv.NavierStokesTransport({}, w0.eos, flux, tr), fv.SpeciesTransport(w0.eos, flux, tr)]
    w = Workload(w0.name, w0.mesh, w0.eos, procs, w0.petscfv_type, w0.limiter, w0.U, w0.description)
    phys, keep = w.physics()
    F, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    return F, w


DK = np.linspace(2e-5, 1.2e-4, 5)


def test_equal_diffusivities_give_the_scalar_residual():
    Fv, w = _rhs("species3d_ns5", np.full(5, 7e-5))
    Fs, _ = _rhs("species3d_ns5", 7e-5)
    assert np.array_equal(Fv, Fs)


@pytest.mark.parametrize("k", range(5))
def test_species_k_uses_its_own_diffusivity(k):
    Fv, w = _rhs("species3d_ns5", DK)
    Fs, _ = _rhs("species3d_ns5", float(DK[k]))
    ne = w.mesh.dim + 2
    assert np.array_equal(Fv[:, ne + k], Fs[:, ne + k])
    assert not np.array_equal(Fv[:, 1], Fs[:, 1])  # the energy flux sums over every species


def test_energy_residual_is_affine_in_the_diffusivities():
    F0, w = _rhs("species3d_ns5", np.zeros(5))
    Fv, _ = _rhs("species3d_ns5", DK)
    acc = F0[:, 1].copy()
    for k in range(5):
        e = np.zeros(5)
        e[k] = DK[k]
        acc += _rhs("species3d_ns5", e)[0][:, 1] - F0[:, 1]
    np.testing.assert_allclose(Fv[:, 1], acc, rtol=1e-10, atol=1e-10 * np.abs(Fv[:, 1]).max())


def test_diffusivity_count_must_match_the_species():
    with pytest.raises(ValueError, match="number of species"):
        _rhs("species3d_ns5", np.ones(4))
