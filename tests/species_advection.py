"""The reference's species advection convergence test (tests/unitTests/finiteVolume/
compressibleFlowSpeciesAdvectionTests.cpp), restated: three species in a perfect gas (gamma 1.4,
R 287) on the square [0, 0.01]^2, uniform flow rho 2, rho E 500000, rho u 8, rho v 0, and mass
fractions advected as a sine wave, rho Y = (0.4 s, 0.6 s, 2 (1 - s / 2)) with
s = (1 + sin(2 pi (x - 4 t) / 0.01)) / 2. AUSM, first order (PetscFV upwind), no transport;
every boundary an EssentialGhost: the ghost cell holds the exact solution at its boundary face's
centroid (DMPlexInsertBoundaryValuesRiemann hands the boundary function the face centroid, and
EssentialGhost without enforceAtFace stores the value as it is, essentialGhost.cpp:5-21); PETSc's
default TS (forward Euler) with dt 5e-5 for 50 steps; 5, 10, 20 and 40 cells per side. The error norms are
the SolutionErrorMonitor's per-component L2 (root mean square over the cells) and Linf; the expected
orders are 1 for the three species within the ConvergenceTester's 0.2, and the Euler components are
reproduced exactly (the reference expects NaN slopes: zero error).
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

DT, STEPS, LEVELS, N0, SIDE = 5e-5, 50, 4, 5, 0.01
EXPECTED = [1.0, 1.0, 1.0]


def exact(x, t):
    s = (1.0 + np.sin(2.0 * np.pi * (x - 4.0 * t) / SIDE)) / 2.0
    U = np.zeros((len(x), 7))
    U[:, 0], U[:, 1], U[:, 2], U[:, 3] = 2.0, 500000.0, 8.0, 0.0
    U[:, 4] = 2 * .2 * s
    U[:, 5] = 2 * .3 * s
    U[:, 6] = 2 * (1 - .5 * s)
    return U


def workload(level):
    from ablate_b200 import fv
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    n = N0 * 2 ** level
    mesh = box_mesh((n, n), upper=(SIDE, SIDE), order="morton")
    eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0}, ["O2", "H2O", "N2"])
    flux = fv.Ausm()
    procs = [fv.NavierStokesTransport({"cfl": 0.25}, eos, flux), fv.SpeciesTransport(eos, flux)]
    U = exact(mesh.cell_centroid[:, 0], 0.0)
    return Workload("species advection", mesh, eos, procs, "upwind", "none", U, "species advection"), SIDE / n


def ghost_face_x(mesh):
    """For every boundary ghost cell (in index order), x of the centroid of its one face."""
    ghost = np.flatnonzero(mesh.cell_kind == L.CELL_BOUNDARY)
    fc = mesh.face_cells
    x = {}
    for side in (0, 1):
        g = mesh.cell_kind[fc[:, side]] == L.CELL_BOUNDARY
        x.update(zip(fc[g, side].tolist(), mesh.face_centroid[g, 0].tolist()))
    return ghost, np.array([x[c] for c in ghost.tolist()])


def march(w, rhs):
    """50 forward-Euler steps; before every evaluation the ghost cells take the exact solution at
    their face centroid and the current time. rhs(t, U) returns the residual. Returns the final state."""
    ghost, xg = ghost_face_x(w.mesh)
    U = w.U.copy()
    t = 0.0
    for _ in range(STEPS):
        U[ghost] = exact(xg, t)
        U = U + DT * rhs(t, U)
        t += DT
    U[ghost] = exact(xg, t)
    return U, t


def errors(w, U, t):
    own = w.mesh.cell_kind == L.CELL_OWNED
    e = (U - exact(w.mesh.cell_centroid[:, 0], t))[own]
    return np.sqrt((e * e).mean(0)), np.abs(e).max(0)


def slopes(hs, norms):
    lh = np.log10(np.asarray(hs))
    return np.array([np.polyfit(lh, np.log10(np.asarray(norms)[:, b]), 1)[0] for b in range(np.asarray(norms).shape[1])])
