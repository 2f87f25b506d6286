"""Any species count. The kernels are compiled for a few exact counts (0, 2, 3 in 2D; 0, 2, 5 and 9 in
3D), for 16 species (RHS, aux update and tangent, unrolled), for 64 species in 3D (RHS, aux update and
tangent, loops over the state components at run time) and for a capacity of 128 species (RHS and aux
update, run-time loops); a count without an instance of its own runs in
the smallest instance that holds it, its species after zero-state padding species, and every entry point
of the RHS and its derivatives translates the rows (the species padding in ablate_b200/csrc/fv.cu).
ABL_FV_SPECIES_INSTANCE at create asks for a larger instance than needed, so that an exact count can be
run padded and compared with itself.

Checked: the RHS at 1, 4, 7 and 12 synthetic NASA-7 species and at the 53 species of the reference's
gri30 mechanism against the oracle (1e-12); the RHS, JVP and VJP of 5 species padded into the 9-species
instance, its RHS and JVP padded into the 16- and 64-species instances and its RHS padded into the
128-species one, against the exact 5-species instance; the refusals of the derivatives an instance does
not compile; the VJP as the transpose of the JVP on padded counts; the JVP of 12 species and of gri30's
53 against central differences; the reference's 1D three-species diffusion convergence test on the
device.
"""
import os

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux
from oracle import oracle as orc
from tests import rhs_cases as R

pytestmark = pytest.mark.gpu


def _solver(w, instance=None):
    old = os.environ.get("ABL_FV_SPECIES_INSTANCE")
    if instance is None:
        os.environ.pop("ABL_FV_SPECIES_INSTANCE", None)
    else:
        os.environ["ABL_FV_SPECIES_INSTANCE"] = str(instance)
    try:
        s = w.solver()
    finally:
        if old is None:
            os.environ.pop("ABL_FV_SPECIES_INSTANCE", None)
        else:
            os.environ["ABL_FV_SPECIES_INSTANCE"] = old
    s.SetAux(initial_aux(w))
    return s


@pytest.mark.parametrize("name", ["species3d_ns1", "species3d_ns4", "species3d_ns7", "species3d_ns12", "gri30_box3d"])
def test_rhs_of_any_species_count_matches_the_oracle(name):
    w = R.case(name)
    phys, keep = w.physics()
    F_ref, aux_ref = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    s = _solver(w)
    F = np.zeros_like(w.U)
    s.ComputeRHSFunction(0.0, w.U, F, L.PRECISION_FP64)
    assert s.Status() == L.OK
    aux = s.GetAux()
    s.close()
    owned = w.mesh.cell_kind == L.CELL_OWNED
    assert np.all(F[~owned] == 0.0)
    np.testing.assert_allclose(aux, aux_ref, rtol=1e-12, atol=1e-9)
    for block, e in R.block_errors(F, F_ref, owned, 2 + w.mesh.dim).items():
        assert e <= 1e-12, f"{name} {block}: {e:.3e}"


def _derivatives(s, w, seed, jvp=True, vjp=True):
    rng = np.random.default_rng(seed)
    F = np.zeros_like(w.U)
    s.ComputeRHSFunction(0.0, w.U, F, L.PRECISION_FP64)
    dU = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0) * 1e-3
    dF = np.zeros_like(w.U)
    Fb = rng.standard_normal(w.U.shape)
    Ub = np.zeros_like(w.U)
    if jvp:
        s.ComputeJVP(0.0, w.U, dU, dF)
    else:
        with pytest.raises(L.AblateError) as e:
            s.ComputeJVP(0.0, w.U, dU, dF)
        assert e.value.code == L.ERR_UNSUPPORTED
    if vjp:
        s.ComputeVJP(0.0, w.U, Fb, Ub)
    else:
        with pytest.raises(L.AblateError) as e:
            s.ComputeVJP(0.0, w.U, Fb, Ub)
        assert e.value.code == L.ERR_UNSUPPORTED
    assert s.Status() == L.OK
    return [F] + ([dF] if jvp else []) + ([Ub] if vjp else [])


@pytest.mark.parametrize("instance,jvp,vjp", [(9, True, True), (16, True, False), (64, True, False), (128, False, False)])
def test_padded_instance_equals_the_exact_instance(instance, jvp, vjp):
    # five species have an instance of their own; run padded they must give the same RHS and the same
    # derivatives where the instance compiles them (the others are refused with ERR_UNSUPPORTED)
    w = R.case("species3d_ns5")
    exact, padded = _solver(w), _solver(w, instance)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    allc = np.ones_like(owned)
    F, dF, Ub = _derivatives(exact, w, 3)
    a_all = [F] + ([dF] if jvp else []) + ([Ub] if vjp else [])
    b_all = _derivatives(padded, w, 3, jvp, vjp)
    what = ["rhs"] + (["jvp"] if jvp else []) + (["vjp"] if vjp else [])
    rows = [owned] + ([owned] if jvp else []) + ([allc] if vjp else [])
    assert len(a_all) == len(b_all) == len(what)
    for a, b, r, wh in zip(a_all, b_all, rows, what):
        for block, e in R.block_errors(b, a, r, 5).items():
            assert e <= 1e-13, f"{wh} {block} in the {instance}-species instance: {e:.3e}"
    exact.close()
    padded.close()


@pytest.mark.parametrize("name", ["species3d_ns4", "species3d_ns7"])
def test_vjp_is_the_transpose_of_the_jvp_for_padded_counts(name):
    # four species run in the 5-species instance, seven in the 9-species one
    w = R.case(name)
    s = _solver(w)
    rng = np.random.default_rng(11)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    v = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0) * 1e-4
    v[~owned] = 0.0  # directions on owned rows (ghosts are boundary data)
    Jv = s.ComputeJVP(0.0, w.U, v, np.zeros_like(w.U))
    u = rng.standard_normal(w.U.shape)
    u[~owned] = 0.0
    JTu = s.ComputeVJP(0.0, w.U, u, np.zeros_like(w.U))
    s.close()
    lhs, rhs = float(np.sum(u * Jv)), float(np.sum(JTu * v))
    scale = float(np.sum(np.abs(u * Jv)))
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)


def test_jvp_of_a_count_in_the_16_species_instance_matches_finite_differences():
    # twelve species run in the 16-species instance: the tangent against a central difference of the RHS
    w = R.case("species3d_ns12")
    s = _solver(w)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    rng = np.random.default_rng(5)
    v = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)
    v[~owned] = 0.0
    Jv = s.ComputeJVP(0.0, w.U, v, np.zeros_like(w.U))
    eps = 1e-6
    Fp, Fm = np.zeros_like(w.U), np.zeros_like(w.U)
    s.ComputeRHSFunction(0.0, w.U + eps * v, Fp, L.PRECISION_FP64)
    s.ComputeRHSFunction(0.0, w.U - eps * v, Fm, L.PRECISION_FP64)
    assert s.Status() == L.OK
    with pytest.raises(L.AblateError) as e:
        s.ComputeVJP(0.0, w.U, v, np.zeros_like(w.U))
    assert e.value.code == L.ERR_UNSUPPORTED
    s.close()
    fd = (Fp - Fm) / (2 * eps)
    assert np.linalg.norm(Jv[owned] - fd[owned]) <= 1e-5 * np.linalg.norm(fd[owned])


def test_jvp_of_gri30_in_the_64_species_instance_matches_finite_differences():
    # the 53 species of gri30 run in the 64-species instance: the tangent against a central difference
    w = R.case("gri30_box3d")
    s = _solver(w)
    owned = w.mesh.cell_kind == L.CELL_OWNED
    rng = np.random.default_rng(5)
    v = rng.standard_normal(w.U.shape) * np.abs(w.U).mean(0)
    v[~owned] = 0.0
    Jv = s.ComputeJVP(0.0, w.U, v, np.zeros_like(w.U))
    eps = 1e-6
    Fp, Fm = np.zeros_like(w.U), np.zeros_like(w.U)
    s.ComputeRHSFunction(0.0, w.U + eps * v, Fp, L.PRECISION_FP64)
    s.ComputeRHSFunction(0.0, w.U - eps * v, Fm, L.PRECISION_FP64)
    assert s.Status() == L.OK
    s.close()
    fd = (Fp - Fm) / (2 * eps)
    assert np.all(np.isfinite(Jv))
    assert np.linalg.norm(Jv[owned] - fd[owned]) <= 1e-6 * np.linalg.norm(fd[owned])


def test_stepping_entry_points_need_a_count_with_its_own_instance():
    w = R.case("species3d_ns4")
    s = _solver(w)
    import torch
    U = torch.from_numpy(w.U).cuda()
    with pytest.raises(L.AblateError) as e:
        s.FillGhostsDevice(U.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert e.value.code == L.ERR_UNSUPPORTED
    s.close()


@pytest.mark.parametrize("rho,vector", [(1.0, False), (2.0, True)])
def test_device_1d_species_diffusion_converges_at_the_reference_order(rho, vector):
    # the reference's 1D three-species diffusion test (compressibleFlowSpeciesDiffusionTests.cpp): three
    # species in 1D run padded in the 16-species instance; the device march equals the oracle's
    from tests import species_diffusion as SD
    hs, l2, li = [], [], []
    for level in SD.LEVELS:
        w, h = SD.workload(level, rho, vector)
        s = _solver(w)
        aux = initial_aux(w)

        def rhs(U):
            F = np.zeros_like(U)
            s.ComputeRHSFunction(0.0, U, F, L.PRECISION_FP64)
            return F

        U, t = SD.march(w, rhs, rho)
        assert s.Status() == L.OK
        s.close()
        phys, keep = w.physics()
        U_ref, _ = SD.march(w, lambda U: orc.rhs(w.mesh, phys, U, aux)[0], rho)
        own = w.mesh.cell_kind == L.CELL_OWNED
        assert np.linalg.norm(U[own] - U_ref[own]) <= 1e-12 * np.linalg.norm(U_ref[own])
        a, b = SD.errors(w, U, t, rho)
        assert np.all(b[:3] == 0.0), b
        hs.append(h)
        l2.append(a)
        li.append(b)
    l2, li = np.array(l2), np.array(li)
    for c, order in SD.EXPECTED.items():
        assert abs(SD.slope(hs, l2[:, c]) - order) <= 0.2, (c, SD.slope(hs, l2[:, c]))
        assert abs(SD.slope(hs, li[:, c]) - order) <= 0.2, (c, SD.slope(hs, li[:, c]))
