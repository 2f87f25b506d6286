"""The reference-side drop-in: the B200Rhs process (ablate_b200/reference_process/b200Rhs.cpp), a
finiteVolume::processes::Process that registers an RHSArbitraryFunction computing the RHS through the C
ABI. It is compiled here with g++ against stand-ins of the reference interfaces it uses
(tests/reference_shim: Process, FiniteVolumeSolver::RegisterRHSFunction, the EOS / flux calculator /
transport classes, a PETSc Vec) and linked with the product library, by tests/reference_process_check.cpp.

CPU: the mapping of the reference's configuration objects to abl_physics_desc, the registration, and the
rejection of configurations without a device counterpart. GPU: one RHS through the registered function
pointer (the stand-in solver's ComputeRHSFunction calls it on locX / locF) against the oracle.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200.workloads import initial_aux

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    if not L.LIB_PATH.exists():
        pytest.skip("the product library is not built")
    exe = tmp_path_factory.mktemp("adapter") / "reference_process_check"
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", str(ROOT / "tests" / "reference_shim"), "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "ablate_b200" / "reference_process"), str(ROOT / "tests" / "reference_process_check.cpp"),
                    str(ROOT / "ablate_b200" / "reference_process" / "b200Rhs.cpp"), "-L", str(L.LIB_PATH.parent), "-lablate_fv",
                    f"-Wl,-rpath,{L.LIB_PATH.parent}", "-o", str(exe)], check=True)
    return exe


def _fields(line):
    name, *rest = line.split()
    return name, dict(kv.split("=", 1) for kv in rest)


def test_reference_objects_map_to_the_descriptor(driver):
    out = subprocess.run([str(driver), "map"], capture_output=True, text=True, check=True).stdout.splitlines()
    rows = dict(_fields(l) for l in out if "=" in l)
    ns = rows["ns_ausmpup_constant"]
    assert (int(ns["eos"]), float(ns["gamma"]), float(ns["r_gas"])) == (L.EOS_PERFECT_GAS, 1.4, 287.0)
    assert (int(ns["flux"]), float(ns["minf"]), float(ns["pgs_alpha"])) == (L.FLUX_AUSMPUP, 0.3, 1.0)
    assert (int(ns["recon"]), int(ns["limiter"])) == (L.RECON_LEASTSQUARES, L.LIMITER_MINMOD)
    # the Constant model's values come from its own transport functions
    assert (int(ns["transport"]), float(ns["k"]), float(ns["mu"])) == (L.TRANSPORT_CONSTANT, 0.0252, 1.8e-5)
    assert (int(ns["species_advection"]), int(ns["species_diffusion"])) == (0, 0)
    sp = rows["species_ausm_upwind"]
    assert (int(sp["n_species"]), int(sp["flux"]), int(sp["recon"]), int(sp["transport"])) == (2, L.FLUX_AUSM, L.RECON_UPWIND, L.TRANSPORT_NONE)
    assert (int(sp["diffusion"]), int(sp["species_advection"])) == (0, 1)
    tc = rows["tchem_average_vector_diff"]
    assert (int(tc["eos"]), int(tc["n_species"]), int(tc["flux"]), int(tc["limiter"])) == (L.EOS_NASA7, 3, L.FLUX_AVERAGE, L.LIMITER_VANLEER)
    # one diffusivity per species selects the VariableDiffusionCoefficient fluxes; molar masses by species name
    assert (tc["species_diff"], tc["nasa7"], float(tc["mw0"]), int(tc["compact"])) == ("set", "set", 31.998, 1)
    rs = rows["riemann_sutherland"]
    assert (int(rs["flux"]), int(rs["transport"]), int(rs["limiter"])) == (L.FLUX_RIEMANN, L.TRANSPORT_SUTHERLAND, L.LIMITER_SIN)
    assert int(rows["off"]["flux"]) == L.FLUX_OFF
    assert "registered 1" in out
    assert "rejected 2" in out


def _write_case(tmp_path, w):
    m = w.mesh
    shift = m.face_shift
    p = tmp_path / "mesh.bin"
    with open(p, "wb") as f:
        np.array([m.dim, m.n_cells, m.n_faces, shift is not None, 1, 1], dtype=np.int32).tofile(f)
        np.ascontiguousarray(m.face_cells, dtype=np.int32).tofile(f)
        for a in (m.face_normal, m.face_centroid, m.cell_centroid, m.cell_volume):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.ascontiguousarray(m.cell_kind, dtype=np.uint8).tofile(f)
        if shift is not None:
            np.ascontiguousarray(shift, dtype=np.float64).tofile(f)
    s = tmp_path / "state.bin"
    np.ascontiguousarray(w.U, dtype=np.float64).tofile(s)
    return p, s


@pytest.mark.skipif(L.device_count() > 0, reason="checks the no-device path")
def test_initialize_reports_a_missing_device(driver, tmp_path):
    from ablate_b200 import workloads
    mesh, state = _write_case(tmp_path, workloads.tgv3d(4))
    r = subprocess.run([str(driver), "rhs", str(mesh), str(state), str(tmp_path / "F.bin"), "ausmpup", "minmod", "0.0252", "1.8e-5"],
                       capture_output=True, text=True)
    assert r.returncode == 3 and "no CUDA device" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name,flux,limiter", [("tgv3d", "ausmpup", "minmod"), ("box2d", "ausm", "vanleer")])
def test_rhs_through_the_registered_function_matches_the_oracle(driver, tmp_path, name, flux, limiter):
    from ablate_b200 import fv, workloads
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    from oracle import oracle as orc
    from tests import rhs_cases as R
    if name == "tgv3d":
        w = workloads.tgv3d(8)
        k, mu = w.processes[0].transport.k, w.processes[0].transport.mu
    else:
        base = R.case("box2d_ausm_minmod_const")
        k, mu = 0.025, 1.8e-5
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0})
        w = Workload(name, base.mesh, eos, [fv.NavierStokesTransport({}, eos, fv.Ausm(), fv.Constant(k=k, mu=mu))], "leastsquares", limiter,
                     base.U, name)
    mesh, state = _write_case(tmp_path, w)
    out = tmp_path / "F.bin"
    r = subprocess.run([str(driver), "rhs", str(mesh), str(state), str(out), flux, limiter, repr(k), repr(mu)], capture_output=True, text=True)
    assert r.returncode == 0 and "rhs ok" in r.stdout, r.stdout + r.stderr
    F = np.fromfile(out, dtype=np.float64).reshape(w.U.shape)
    phys, keep = w.physics()
    F_ref, _ = orc.rhs(w.mesh, phys, w.U, initial_aux(w))
    owned = w.mesh.cell_kind == L.CELL_OWNED
    for block, e in R.block_errors(F, F_ref, owned, 2 + w.mesh.dim).items():
        assert e <= 1e-12, (name, block, e)
