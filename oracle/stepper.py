"""CPU restatement of the steps around the RHS in an explicit time step.

Test infrastructure: the oracle the device time stepping is checked against. Nothing here is a product
path; the product runs these steps as CUDA kernels (ablate_b200/csrc/fv_step.cuh).

  fill_ghosts        the Ghost / EssentialGhost update functions DMPlexInsertBoundaryValuesRiemann
                     applies before every RHS (src/solver/solver.cpp:50-102,
                     src/finiteVolume/boundaryConditions/ghost.cpp:17-28, essentialGhost.cpp:5-22)
  cfl_dt             NavierStokesTransport::ComputeCflTimeStep (navierStokesTransport.cpp:209-278) with the
                     minimum cell radius of FiniteVolumeSolver (finiteVolumeSolver.cpp:172-218)
  normalize_species  SpeciesTransport::NormalizeSpecies (speciesTransport.cpp:343-403)
  fill_ghosts_tangent, fill_ghosts_adjoint
                     derivative of the ghost fill and its transpose (no reference counterpart: the
                     reference has no adjoint); the transpose sums per interior cell in ascending ghost order
  pressure_functional  J = sum_j w_j p(U_c_j) and, for a perfect gas, dJ/dU in closed form
                     (p = (gamma - 1)(rho E - |rho u|^2 / (2 rho)), src/eos/perfectGas.cpp:49-197)
  march_functional   J after a fixed-step march (for finite differences of the marched functional)
  euler_step, ssprk3_step, integrate
                     explicit steps; integrate chooses steps as AdaptPhysics does (the CFL step times
                     the safety factor, src/solver/adaptPhysics.cpp:3-24) and ends exactly at the final
                     time (TS_EXACTFINALTIME_MATCHSTEP, src/solver/timeStepper.cpp:37). Checked against
                     the reference's shock-tube profiles (compressibleShockTubeTests.cpp:210+).
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

from . import oracle as orc

OUTFLOW, DIRICHLET, SLIP_WALL, NOSLIP_WALL = 0, 1, 2, 3


def ghost_pairs(mesh):
    """(ghost cells, their interior neighbours, unit normals out of the domain)."""
    fc = mesh.face_cells
    kind = mesh.cell_kind
    g_is_r = kind[fc[:, 1]] == L.CELL_BOUNDARY
    g_is_l = kind[fc[:, 0]] == L.CELL_BOUNDARY
    n = mesh.face_normal / np.linalg.norm(mesh.face_normal, axis=1, keepdims=True)
    ghosts = np.concatenate([fc[g_is_r, 1], fc[g_is_l, 0]])
    inner = np.concatenate([fc[g_is_r, 0], fc[g_is_l, 1]])
    normal = np.concatenate([n[g_is_r], -n[g_is_l]])
    return ghosts, inner, normal


def fill_ghosts(mesh, U, table, cell_bc=None):
    """table: list of (kind, value or None, enforce_at_face); cell_bc[c] names the entry of ghost c."""
    ghosts, inner, normal = ghost_pairs(mesh)
    dim = mesh.dim
    for j in range(ghosts.size):
        g, i = ghosts[j], inner[j]
        kind, value, enforce = table[0 if cell_bc is None else cell_bc[g]]
        u = U[i].copy()
        if kind == DIRICHLET:
            v = np.asarray(value, float)[:U.shape[1]]
            u = 2.0 * v - u if enforce else v.copy()
        elif kind == SLIP_WALL:
            mn = float(np.dot(u[2:2 + dim], normal[j, :dim]))
            u[2:2 + dim] -= 2.0 * mn * normal[j, :dim]
        elif kind == NOSLIP_WALL:
            u[2:2 + dim] = -u[2:2 + dim]
        U[g] = u
    return U


def fill_ghosts_tangent(mesh, dU, table, cell_bc=None):
    """Derivative of fill_ghosts with respect to the interior rows (the condition values held fixed)."""
    ghosts, inner, normal = ghost_pairs(mesh)
    dim = mesh.dim
    for j in range(ghosts.size):
        g, i = ghosts[j], inner[j]
        kind, value, enforce = table[0 if cell_bc is None else cell_bc[g]]
        u = dU[i].copy()
        if kind == DIRICHLET:
            u = -u if enforce else np.zeros_like(u)
        elif kind == SLIP_WALL:
            mn = float(np.dot(u[2:2 + dim], normal[j, :dim]))
            u[2:2 + dim] -= 2.0 * mn * normal[j, :dim]
        elif kind == NOSLIP_WALL:
            u[2:2 + dim] = -u[2:2 + dim]
        dU[g] = u
    return dU


def fill_ghosts_adjoint(mesh, Ub, table, cell_bc=None):
    """Transpose of fill_ghosts on adjoint rows, in place: returns (Ub, vbar[n_bc][nc]). Per interior cell
    the ghosts' terms are summed in ascending ghost order first, then added to the cell's row."""
    ghosts, inner, normal = ghost_pairs(mesh)
    dim = mesh.dim
    nc = Ub.shape[1]
    vbar = np.zeros((len(table), nc))
    acc = {}
    for j in np.lexsort((ghosts, inner)):
        g, i = ghosts[j], inner[j]
        b = 0 if cell_bc is None else cell_bc[g]
        kind, value, enforce = table[b]
        lg = Ub[g].copy()
        Ub[g] = 0.0
        a = acc.setdefault(i, np.zeros(nc))
        if kind == DIRICHLET:
            vbar[b] += 2.0 * lg if enforce else lg
            if enforce:
                a -= lg
        elif kind == SLIP_WALL:
            mn = float(np.dot(lg[2:2 + dim], normal[j, :dim]))
            lg[2:2 + dim] -= 2.0 * mn * normal[j, :dim]
            a += lg
        elif kind == NOSLIP_WALL:
            lg[2:2 + dim] = -lg[2:2 + dim]
            a += lg
        else:
            a += lg
    for i, a in acc.items():
        Ub[i] += a
    return Ub, vbar


def pressure_functional(mesh, physics, U, cells, weights, gamma=None):
    """J = sum_j w_j p(U[c_j]) through the oracle EOS; with gamma (perfect gas), also dJ/dU."""
    Uc = np.ascontiguousarray(U[cells])
    T = orc.eos(physics, mesh.dim, L.PROP_TEMPERATURE, Uc, np.full(len(cells), 300.0))[:, 0]
    p = orc.eos(physics, mesh.dim, L.PROP_PRESSURE, Uc, T)[:, 0]
    J = float(np.dot(weights, p))
    if gamma is None:
        return J, None
    G = np.zeros_like(U)
    rho = Uc[:, 0]
    vel = Uc[:, 2:2 + mesh.dim] / rho[:, None]
    G[cells, 0] = weights * (gamma - 1.0) * 0.5 * (vel ** 2).sum(1)
    G[cells, 1] = weights * (gamma - 1.0)
    G[cells, 2:2 + mesh.dim] = -(weights * (gamma - 1.0))[:, None] * vel
    return J, G


def march_functional(mesh, physics, U, dt, n_steps, table, cell_bc, cells, weights, step="ssprk3"):
    """J after n_steps fixed steps of size dt from U (the march the device adjoint differentiates)."""
    U = U.copy()
    for _ in range(n_steps):
        U = euler_step(mesh, physics, U, dt, table, cell_bc) if step == "euler" else ssprk3_step(mesh, physics, U, dt, table, cell_bc)
        if step == "euler":
            fill_ghosts(mesh, U, table, cell_bc)
    return pressure_functional(mesh, physics, U, cells, weights)[0]


def min_cell_radius(mesh):
    """Smallest distance from a cell centroid to the centroid of one of its faces."""
    r = np.full(mesh.n_cells, np.inf)
    fc = mesh.face_cells
    shift = mesh.face_shift if mesh.face_shift is not None else np.zeros_like(mesh.face_centroid)
    dL = np.linalg.norm((mesh.face_centroid - mesh.cell_centroid[fc[:, 0]])[:, :mesh.dim], axis=1)
    dR = np.linalg.norm((mesh.face_centroid - shift - mesh.cell_centroid[fc[:, 1]])[:, :mesh.dim], axis=1)
    np.minimum.at(r, fc[:, 0], dL)
    np.minimum.at(r, fc[:, 1], dR)
    return r


def cfl_dt(mesh, physics, U, cfl, alpha=1.0):
    owned = mesh.cell_kind == L.CELL_OWNED
    dim = mesh.dim
    Uo = np.ascontiguousarray(U[owned])
    T = orc.eos(physics, dim, L.PROP_TEMPERATURE, Uo, np.full(Uo.shape[0], 300.0))[:, 0]
    a = orc.eos(physics, dim, L.PROP_SPEED_OF_SOUND, Uo, T)[:, 0]
    vel_sum = np.zeros(Uo.shape[0])
    for d in range(dim):
        vel_sum += np.abs(Uo[:, 2 + d]) / Uo[:, 0]
    dt = cfl * (2.0 * min_cell_radius(mesh)[owned]) / (a / alpha + vel_sum)
    return float(dt.min())


def normalize_species(mesh, U, ns):
    if ns == 0:
        return U
    owned = mesh.cell_kind == L.CELL_OWNED
    ne = U.shape[1] - ns
    for c in np.nonzero(owned)[0]:
        density = U[c, 0]
        rY = U[c, ne:]
        s = 0.0
        for k in range(ns - 1):
            yi = min(1.0, max(0.0, rY[k] / density))
            s += yi
            rY[k] = yi * density
        if s > 1.0:
            for k in range(ns):
                rY[k] = density * ((rY[k] / density) / s)
            rY[ns - 1] = 0.0
        else:
            rY[ns - 1] = density * (1.0 - s)
    return U


def _L(mesh, physics, U, aux, table, cell_bc):
    fill_ghosts(mesh, U, table, cell_bc)
    F, _ = orc.rhs(mesh, physics, U, aux)
    return F


def euler_step(mesh, physics, U, dt, table, cell_bc=None, aux=None):
    owned = (mesh.cell_kind == L.CELL_OWNED)[:, None]
    F = _L(mesh, physics, U, aux, table, cell_bc)
    return np.where(owned, U + dt * F, U)


def ssprk3_step(mesh, physics, U, dt, table, cell_bc=None, aux=None, ns=0):
    """Three-stage SSP Runge-Kutta (Shu-Osher form) on the owned rows, species normalised after."""
    owned = (mesh.cell_kind == L.CELL_OWNED)[:, None]
    U0 = U.copy()
    U1 = U.copy()
    F = _L(mesh, physics, U1, aux, table, cell_bc)
    U1 = np.where(owned, 1.0 * (U0 + dt * F), U1)
    F = _L(mesh, physics, U1, aux, table, cell_bc)
    U1 = np.where(owned, 0.75 * U0 + 0.25 * (U1 + dt * F), U1)
    F = _L(mesh, physics, U1, aux, table, cell_bc)
    U = np.where(owned, (1.0 / 3.0) * U0 + (2.0 / 3.0) * (U1 + dt * F), U1)
    U = normalize_species(mesh, U, ns)
    fill_ghosts(mesh, U, table, cell_bc)
    return U


def match_step(h, t, t_end):
    """Next step so the march ends exactly at t_end without a sliver of a last step (PETSc's
    TS_EXACTFINALTIME_MATCHSTEP with its default factors 1.01 and 2, which TimeStepper selects,
    src/solver/timeStepper.cpp:37): t is the time the step starts from."""
    hmax = t_end - t
    if t < t_end and t + h > t_end:
        h = hmax
    if t < t_end and t + h < t_end and h * 2.0 > hmax:
        h = hmax / 2.0
    if t < t_end and t + h < t_end and h * 1.01 > hmax:
        h = hmax
    return h


def integrate(mesh, physics, U, t_end, cfl, table, cell_bc=None, step="euler", dt0=0.1, ns=0):
    """March to t_end as the reference's TimeStepper does with ts_adapt_type physics: the first step is
    min(dt0, CFL step of the initial state); after every step the next one is the CFL step of the state
    that step started from (the adaptor runs before the solution vector takes the update), adjusted by
    match_step. step "euler" is PETSc's default explicit TS (forward Euler); "ssprk3" the three-stage
    SSP Runge-Kutta. Returns (U, number of steps)."""
    U = U.copy()
    fill_ghosts(mesh, U, table, cell_bc)
    t, n = 0.0, 0
    dt = match_step(min(dt0, cfl_dt(mesh, physics, U, cfl)), t, t_end)
    while t < t_end:
        nxt = cfl_dt(mesh, physics, U, cfl)
        U = euler_step(mesh, physics, U, dt, table, cell_bc) if step == "euler" else ssprk3_step(mesh, physics, U, dt, table, cell_bc, ns=ns)
        t = t_end if t + dt >= t_end or t_end - (t + dt) <= 1e-12 * t_end else t + dt
        n += 1
        dt = match_step(nxt, t, t_end)
    fill_ghosts(mesh, U, table, cell_bc)
    return U, n
