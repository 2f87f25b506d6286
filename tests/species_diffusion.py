"""The reference's 1D species diffusion convergence test (tests/unitTests/finiteVolume/
compressibleFlowSpeciesDiffusionTests.cpp), restated. Three species at rest in [0, 0.1] with
density rho; Y0 diffuses from 0.5 to walls held at 0 (the sine series the test sums, 2000 terms),
Y1 = 0.5 - Y0, Y2 = 0.5; SpeciesTransport with diffusion only (Constant transport k = mu = 0 and the
diffusivity 1e-5, scalar or one per species), no species normalisation.

Boundaries: EssentialGhost with enforceAtFace (twice the exact value at the face centroid minus the
interior value, essentialGhost.cpp:5-21); time stepping: PETSc's TS "rk" default, the Bogacki-Shampine
3(2) tableau (TSRK3BS, no adaptivity), dt 0.5 to t = 15, boundary values at the stage times; 6, 12
and 24 cells. Expected orders: 2.2 for rho Y0 and rho Y1 within 0.2; rho, rho u and rho Y2 exact
(NaN slopes in the reference).

Not ported: the reference's rho E check (order 2.2). Its mock EOS gives the species sensible
enthalpies 1000, 2000 and 3000 J/kg at every temperature. No EOS here has temperature-independent
enthalpies that differ between species. A NASA-7 mixture with them at one temperature leaves that
temperature at the walls, where the enforceAtFace ghosts carry negative rho Y0 that the mixture
clips. So the gas here is a perfect gas with species (zero sensible enthalpies): the energy
diffusion flux vanishes and rho E stays exact.
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

LEN, DIFF = 0.1, 1e-5
DT, T_END, N0, LEVELS = 0.5, 15.0, 3, (1, 2, 3)
EXPECTED = {3: 2.2, 4: 2.2}  # component -> order; the others exact
# Bogacki-Shampine 3(2): stage times and the combinations of earlier stages
RK_C = (0.0, 0.5, 0.75)
RK_A = ((), (0.5,), (0.0, 0.75))
RK_B = (2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0)


def eos():
    from ablate_b200 import fv
    return fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0}, ["sp0", "sp1", "sp2"])


def y0(x, t):
    n = np.arange(1, 2000, dtype=np.float64)[:, None]
    bn = -0.5 * 2.0 * (-1.0 + (-1.0) ** n) / (n * np.pi)
    return (bn * np.sin(n * np.pi * x[None, :] / LEN) * np.exp(-n * n * np.pi * np.pi * DIFF * t / LEN ** 2)).sum(0)


def exact(mix, x, t, rho):
    a = y0(x, t)
    U = np.zeros((len(x), 6))
    U[:, 0] = rho
    U[:, 1] = rho * 717.5 * 300.0  # rho e of a perfect gas at 300 K, at rest
    U[:, 3] = rho * a
    U[:, 4] = rho * (0.5 - a)
    U[:, 5] = rho * 0.5
    return U


def workload(level, rho, vector):
    from ablate_b200 import fv
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    n = N0 * 2 ** level
    mesh = box_mesh((n,), upper=(LEN,))
    mix = eos()
    tr = fv.Constant(k=0.0, mu=0.0, diff=np.full(3, DIFF) if vector else DIFF)
    U = exact(mix, mesh.cell_centroid[:, 0], 0.0, rho)
    return Workload("species diffusion", mesh, mix, [fv.SpeciesTransport(mix, None, tr)], "upwind", "none", U, "1D species diffusion"), LEN / n


def march(w, rhs, rho):
    """RK3BS to t = 15 with dt 0.5; before every stage evaluation the ghosts take twice the exact
    value at their face centroid (the stage time) minus their interior neighbour."""
    from ablate_b200.mesh import ghost_interior_map
    ghost = np.flatnonzero(w.mesh.cell_kind == L.CELL_BOUNDARY)
    inner = ghost_interior_map(w.mesh)
    fc = w.mesh.face_cells
    xf = {}
    for side in (0, 1):
        g = w.mesh.cell_kind[fc[:, side]] == L.CELL_BOUNDARY
        xf.update(zip(fc[g, side].tolist(), w.mesh.face_centroid[g, 0].tolist()))
    xg = np.array([xf[c] for c in ghost.tolist()])

    def with_ghosts(U, t):
        U = U.copy()
        U[ghost] = 2.0 * exact(w.eos, xg, t, rho) - U[inner]
        return U

    U = w.U.copy()
    t = 0.0
    for _ in range(int(round(T_END / DT))):
        ks = []
        for i, c in enumerate(RK_C):
            Ui = U + DT * sum(a * k for a, k in zip(RK_A[i], ks)) if i else U
            ks.append(rhs(with_ghosts(Ui, t + c * DT)))
        U = U + DT * sum(b * k for b, k in zip(RK_B, ks))
        t += DT
    return U, t


def errors(w, U, t, rho):
    own = w.mesh.cell_kind == L.CELL_OWNED
    e = (exact(w.eos, w.mesh.cell_centroid[own, 0], t, rho) - U[own])
    return np.sqrt((e * e).mean(0)), np.abs(e).max(0)


def slope(hs, errs):
    return float(np.polyfit(np.log10(np.asarray(hs)), np.log10(np.asarray(errs)), 1)[0])
