"""The steps around the RHS on the device (ghost-cell boundary values, CFL step, species normalisation,
explicit steps) against the oracle's restatement (oracle/stepper.py), and the reference's shock-tube
profiles reproduced by the device march (tests/golden/shock_tube.json, tolerance 1e-6 as in the
reference's compressibleShockTubeTests.cpp)."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.workloads import initial_aux
from oracle import stepper as S
from tests import rhs_cases as R
from tests.test_oracle_shock_tube import GOLD, primitives, shock_tube

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.device("cuda", 0))


def _table(w, rng):
    nc = w.U.shape[1]
    ref = np.abs(w.U[w.mesh.cell_kind == L.CELL_OWNED]).mean(0)
    return [(S.OUTFLOW, None, False), (S.DIRICHLET, list(ref * 1.1), False), (S.DIRICHLET, list(ref * 0.9), True),
            (S.SLIP_WALL, None, False), (S.NOSLIP_WALL, None, False)][: 5 if nc else 1]


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "box2d_ausmpup_vanleer_suth", "species3d_ns5", "box1d_riemann_upwind"])
def test_ghost_fill_matches_the_oracle(name):
    torch = pytest.importorskip("torch")
    w = R.case(name)
    s = w.solver()
    rng = np.random.default_rng(5)
    table = _table(w, rng)
    cell_bc = rng.integers(0, len(table), w.mesh.n_cells).astype(np.int32)
    s.SetBoundary(table, cell_bc)
    U = w.U.copy()
    U[w.mesh.cell_kind == L.CELL_BOUNDARY] = np.nan
    ref = S.fill_ghosts(w.mesh, U.copy(), table, cell_bc)
    Ud = _dev(torch, U)
    s.FillGhostsDevice(Ud.data_ptr(), torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(Ud.cpu().numpy(), ref)


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "tgv3d_ausmpup_lsq_minmod_visc", "species3d_ns5", "species3d_ns9", "box1d_riemann_upwind"])
def test_cfl_step_matches_the_oracle(name):
    torch = pytest.importorskip("torch")
    w = R.case(name)
    phys, keep = w.physics()
    s = w.solver()
    Ud = _dev(torch, w.U)
    for cfl in (0.5, 0.9):
        dt = s.CflTimeStepDevice(Ud.data_ptr(), cfl, torch.cuda.current_stream().cuda_stream)
        ref = S.cfl_dt(w.mesh, phys, w.U, cfl)
        assert abs(dt - ref) <= 1e-14 * ref, (dt, ref)


@pytest.mark.parametrize("name", ["species3d_ns5", "pgspecies3d_ns2"])
def test_species_normalisation_matches_the_oracle(name):
    torch = pytest.importorskip("torch")
    w = R.case(name)
    s = w.solver()
    ns = len(w.eos.GetSpeciesVariables())
    rng = np.random.default_rng(2)
    U = w.U.copy()
    ne = U.shape[1] - ns
    U[:, ne:] *= rng.uniform(-0.2, 1.6, (U.shape[0], ns))  # out of [0, 1] and not summing to rho
    ref = S.normalize_species(w.mesh, U.copy(), ns)
    Ud = _dev(torch, U)
    import ctypes as C
    L.check(L.lib.abl_fv_normalize_species(s.handle, C.c_void_p(Ud.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    np.testing.assert_array_equal(Ud.cpu().numpy(), ref)


@pytest.mark.parametrize("case", GOLD["cases"], ids=[c["name"] for c in GOLD["cases"]])
def test_device_march_reproduces_the_reference_shock_tube(case):
    torch = pytest.importorskip("torch")
    mesh, U, table, cell_bc, eos, procs = shock_tube(case)
    s = fv.FiniteVolumeSolver(mesh, eos, procs, "upwind", "none")
    s.SetBoundary(table, cell_bc)
    Ud = _dev(torch, U)
    n = s.IntegrateDevice(Ud.data_ptr(), case["maxTime"], case["cfl"], L.STEP_EULER, L.PRECISION_FP64, 0.1,
                          torch.cuda.current_stream().cuda_stream)
    assert s.Status() == L.OK
    got = primitives(mesh, Ud.cpu().numpy())
    for k, ref in case["expected"].items():
        np.testing.assert_allclose(got[k], ref, rtol=0, atol=1e-6, err_msg=k)
    phys, keep = fv.make_physics(eos, procs, "upwind", "none")
    Uo, no = S.integrate(mesh, phys, U, case["maxTime"], case["cfl"], table, cell_bc)
    assert n == no
    np.testing.assert_allclose(Ud.cpu().numpy(), Uo, rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "tgv3d_ausmpup_lsq_minmod_visc", "species3d_ns5", "box2d_ausmpup_vanleer_suth"])
@pytest.mark.parametrize("scheme", [L.STEP_EULER, L.STEP_SSPRK3])
def test_explicit_steps_match_the_oracle(name, scheme):
    torch = pytest.importorskip("torch")
    w = R.case(name)
    phys, keep = w.physics()
    s = w.solver()
    aux = initial_aux(w)
    s.SetAux(aux)
    table = [(S.OUTFLOW, None, False)]
    ns = len(w.eos.GetSpeciesVariables())
    dt = 0.2 * S.cfl_dt(w.mesh, phys, w.U, 1.0)
    Ud = _dev(torch, w.U)
    U = w.U.copy()
    for k in range(4):
        s.StepDevice(scheme, 0.0, dt, Ud.data_ptr(), L.PRECISION_FP64, torch.cuda.current_stream().cuda_stream)
        if scheme == L.STEP_EULER:
            U = S.euler_step(w.mesh, phys, U, dt, table, aux=aux)
            U = S.normalize_species(w.mesh, U, ns)
            S.fill_ghosts(w.mesh, U, table)
        else:
            U = S.ssprk3_step(w.mesh, phys, U, dt, table, aux=aux, ns=ns)
    assert s.Status() == L.OK
    got = Ud.cpu().numpy()
    owned = w.mesh.cell_kind == L.CELL_OWNED
    # the increments are what the steps compute: compare them relative to their own size
    inc_ref, inc = U[owned] - w.U[owned], got[owned] - w.U[owned]
    assert np.linalg.norm(inc - inc_ref) <= 1e-10 * np.linalg.norm(inc_ref)


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "species3d_ns5", "tets3d_pg_minmod"])
def test_owned_rows_download_and_upload(name):
    """The owned rows leave and re-enter the device unchanged, in ascending local order (the rank's
    global vector), and an upload touches no other row."""
    torch = pytest.importorskip("torch")
    w = R.case(name)
    s = w.solver()
    owned = w.mesh.cell_kind == L.CELL_OWNED
    Ud = _dev(torch, w.U)
    st = torch.cuda.current_stream().cuda_stream
    np.testing.assert_array_equal(s.DownloadOwnedDevice(Ud.data_ptr(), stream=st), w.U[owned])
    rng = np.random.default_rng(9)
    new = rng.standard_normal((int(owned.sum()), w.U.shape[1]))
    s.UploadOwnedDevice(new, Ud.data_ptr(), st)
    got = Ud.cpu().numpy()
    np.testing.assert_array_equal(got[owned], new)
    np.testing.assert_array_equal(got[~owned], w.U[~owned])
    aux = initial_aux(w)
    Ad = _dev(torch, aux)
    np.testing.assert_array_equal(s.DownloadOwnedDevice(Ad.data_ptr(), aux.shape[1], st), aux[owned])


@pytest.mark.parametrize("name", ["sod2d_ausm_upwind", "species3d_ns5"])
@pytest.mark.parametrize("scheme", [L.STEP_EULER, L.STEP_SSPRK3])
def test_device_cfl_steps_match_host_cfl_steps(name, scheme):
    """Steps whose CFL step stays on the device reproduce the host loop (CFL step read back, then the
    step) bit for bit, and the device clock sums the steps."""
    torch = pytest.importorskip("torch")
    w = R.case(name)
    # one handle per march: the mixture EOS keeps its last temperatures as the next solve's guess
    sh, sd = w.solver(), w.solver()
    sh.SetAux(initial_aux(w))
    sd.SetAux(initial_aux(w))
    st = torch.cuda.current_stream().cuda_stream
    Uh = _dev(torch, w.U)
    Ud = _dev(torch, w.U)
    t = torch.zeros(1, dtype=torch.float64, device=Ud.device)
    total = 0.0
    for _ in range(4):
        sh.FillGhostsDevice(Uh.data_ptr(), st)
        dt = sh.CflTimeStepDevice(Uh.data_ptr(), 0.5, st)
        sh.StepDevice(scheme, total, dt, Uh.data_ptr(), L.PRECISION_FP64, st)
        total += dt
        sd.StepCflDevice(scheme, 0.5, Ud.data_ptr(), L.PRECISION_FP64, t.data_ptr(), st)
    assert sh.Status() == L.OK and sd.Status() == L.OK
    assert torch.equal(Uh, Ud)
    assert float(t.item()) == total
