"""The reference's 1D conduction convergence test (tests/unitTests/finiteVolume/
compressibleFlowEulerDiffusionTests.cpp, case "conduction"), restated: a perfect gas (gamma 1.4, R 1)
at rest with rho 1 on [0, 0.1], initially at 400 K, walls held at 300 K; conduction only (OffFlux for
the advection, Constant transport k 0.3, mu 0), so T follows the heat equation with
alpha = k / (rho cv), whose exact solution is the sine series the test sums (2000 terms). The ghost
cells hold twice the wall state minus the interior state (PhysicsBoundary_Euler: the wall value on
the face); PETSc's default TS (forward Euler) with dt 6.25e-6 for 600 steps; 3, 6 and 12 cells. The
errors are root mean squares and maxima over the cells; the expected orders are 2.25 for rho E within
0.2, and rho and rho u stay exact (the reference expects NaN slopes).
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

GAMMA, R, K, RHO, T_INIT, T_WALL, LEN = 1.4, 1.0, 0.3, 1.0, 400.0, 300.0, 0.1
DT, STEPS, N0, LEVELS = 6.25e-6, 600, 3, 3
EXPECTED = 2.25


def temperature(x, t):
    cv = GAMMA * R / (GAMMA - 1) - R
    alpha = K / (RHO * cv)
    n = np.arange(1, 2000, dtype=np.float64)[:, None]
    bn = -(T_INIT - T_WALL) * 2.0 * (-1.0 + (-1.0) ** n) / (n * np.pi)
    return (bn * np.sin(n * np.pi * x[None, :] / LEN) * np.exp(-n * n * np.pi * np.pi * alpha * t / LEN ** 2)).sum(0) + T_WALL


def state(T):
    p = RHO * R * T
    U = np.zeros((len(T), 3))
    U[:, 0] = RHO
    U[:, 1] = RHO * p / ((GAMMA - 1.0) * RHO)
    return U


def workload(level):
    from ablate_b200 import fv
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    n = N0 * 2 ** level
    mesh = box_mesh((n,), upper=(LEN,))
    eos = fv.PerfectGas({"gamma": GAMMA, "Rgas": R})
    procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, fv.OffFlux(), fv.Constant(k=K))]
    U = state(temperature(mesh.cell_centroid[:, 0], 0.0))
    return Workload("conduction", mesh, eos, procs, "upwind", "none", U, "1D conduction"), LEN / n


def march(w, rhs):
    """600 forward-Euler steps, the ghost cells set to twice the wall state minus their interior
    neighbour before every evaluation. rhs(U) returns the residual."""
    from ablate_b200.mesh import ghost_interior_map
    ghost = np.flatnonzero(w.mesh.cell_kind == L.CELL_BOUNDARY)
    inner = ghost_interior_map(w.mesh)
    wall = state(np.array([T_WALL]))[0]
    U = w.U.copy()
    for _ in range(STEPS):
        U[ghost] = 2.0 * wall - U[inner]
        U = U + DT * rhs(U)
    return U, STEPS * DT


def errors(w, U, t):
    own = w.mesh.cell_kind == L.CELL_OWNED
    e = (state(temperature(w.mesh.cell_centroid[own, 0], t)) - U[own])
    return np.sqrt((e * e).mean(0)), np.abs(e).max(0)


def slope(hs, errs):
    return float(np.polyfit(np.log10(np.asarray(hs)), np.log10(np.asarray(errs)), 1)[0])
