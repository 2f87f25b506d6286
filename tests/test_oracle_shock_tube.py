"""The oracle's explicit march reproduces the reference's 1D shock-tube profiles
(tests/unitTests/finiteVolume/compressibleShockTubeTests.cpp:210+, fixture tests/golden/shock_tube.json)
to the reference's own tolerance, 1e-6 on rho, u and e. This pins the first-order AUSM RHS, the
ghost-cell boundary values, the CFL step and the step choice of the reference's TimeStepper at once."""
import json
from pathlib import Path

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from ablate_b200.mesh import box_mesh
from oracle import stepper as S

GOLD = json.loads((Path(__file__).parent / "golden" / "shock_tube.json").read_text())


def shock_tube(case):
    """Mesh, initial state, boundary table and physics of one reference case."""
    ic = case["initial"]
    g = ic["gamma"]
    mesh = box_mesh((case["nx"],), lower=(0.0,), upper=(ic["length"],))

    def state(side):
        rho, u, p = ic["rho" + side], ic["u" + side], ic["p" + side]
        e = p / ((g - 1.0) * rho)
        return [rho, rho * (e + 0.5 * u * u), rho * u]

    left = mesh.cell_centroid[:, 0] < ic["length"] / 2.0
    U = np.zeros((mesh.n_cells, 3))
    U[left] = state("L")
    U[~left] = state("R")
    # the reference's ghost function returns the left state for faces left of the middle
    table = [(S.DIRICHLET, state("L"), False), (S.DIRICHLET, state("R"), False)]
    ghosts, inner, normal = S.ghost_pairs(mesh)
    cell_bc = np.zeros(mesh.n_cells, np.int32)
    cell_bc[ghosts] = np.where(normal[:, 0] < 0, 0, 1)
    eos = fv.PerfectGas({"gamma": g})
    procs = [fv.NavierStokesTransport({"cfl": case["cfl"]}, eos, getattr(fv, case["flux"])())]
    return mesh, U, table, cell_bc, eos, procs


def primitives(mesh, U):
    o = mesh.cell_kind == L.CELL_OWNED
    rho = U[o, 0]
    u = U[o, 2] / rho
    return {"x": mesh.cell_centroid[o, 0], "rho": rho, "u": u, "e": U[o, 1] / rho - 0.5 * u * u}


@pytest.mark.parametrize("case", GOLD["cases"], ids=[c["name"] for c in GOLD["cases"]])
def test_oracle_march_reproduces_the_reference_shock_tube(case):
    mesh, U, table, cell_bc, eos, procs = shock_tube(case)
    phys, keep = fv.make_physics(eos, procs, "upwind", "none")
    Uf, n = S.integrate(mesh, phys, U, case["maxTime"], case["cfl"], table, cell_bc)
    got = primitives(mesh, Uf)
    for k, ref in case["expected"].items():
        np.testing.assert_allclose(got[k], ref, rtol=0, atol=1e-6, err_msg=k)
