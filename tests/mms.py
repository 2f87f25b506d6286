"""Manufactured solutions of the reference's RHS convergence test (compressibleFlowMmsSourceTests.cpp):
smooth 2D Euler fields built from sines and cosines, the source that makes them steady, and the
convergence orders of the residual RHS(U_exact) + S over the central third of the unit square.

The source is the divergence of the exact Euler flux, formed here by complex-step differentiation
(f'(x) = Im f(x + ih) / h, exact to rounding) of the flux of the manufactured fields, rather than from
a closed form.
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

# the reference's four 2D parameter sets: field -> (phi0, phiX, phiY, aPhiX, aPhiY); gamma 1.4, R 287, L 1
LOW = {"rho": (1.0, 0.15, -0.1, 1.0, 0.5), "u": (70.0, 5.0, -7.0, 1.5, 0.6), "v": (90.0, -15.0, -8.5, 0.5, 2.0 / 3.0),
       "p": (1e5, 0.2e5, 0.5e5, 2.0, 1.0)}
HIGH = {"rho": (1.0, 0.15, -0.1, 1.0, 0.5), "u": (800.0, 50.0, -30.0, 1.5, 0.6), "v": (800.0, -75.0, 40.0, 0.5, 2.0 / 3.0),
        "p": (1e5, 0.2e5, 0.5e5, 2.0, 1.0)}
GAMMA = 1.4


def primitives(c, x, y):
    """rho, u, v, p at (x, y) (arrays, real or complex). Which term carries a sine and which a cosine
    follows the reference: rho = r0 + rY cos + rX sin, u = u0 + uY cos + uX sin, v = v0 + vX cos + vY sin,
    p = p0 + pX cos + pY sin."""
    pi = np.pi
    r0, rX, rY, arX, arY = c["rho"]
    u0, uX, uY, auX, auY = c["u"]
    v0, vX, vY, avX, avY = c["v"]
    p0, pX, pY, apX, apY = c["p"]
    rho = r0 + rY * np.cos(arY * pi * y) + rX * np.sin(arX * pi * x)
    u = u0 + uY * np.cos(auY * pi * y) + uX * np.sin(auX * pi * x)
    v = v0 + vX * np.cos(avX * pi * x) + vY * np.sin(avY * pi * y)
    p = p0 + pX * np.cos(apX * pi * x) + pY * np.sin(apY * pi * y)
    return rho, u, v, p


def conserved(c, x, y):
    rho, u, v, p = primitives(c, x, y)
    E = p / ((GAMMA - 1.0) * rho) + 0.5 * (u * u + v * v)
    return np.stack([rho, rho * E, rho * u, rho * v], -1)


def _flux(c, x, y, axis):
    rho, u, v, p = primitives(c, x, y)
    E = p / ((GAMMA - 1.0) * rho) + 0.5 * (u * u + v * v)
    un = u if axis == 0 else v
    return np.stack([rho * un, (rho * E + p) * un, rho * u * un + (p if axis == 0 else 0.0), rho * v * un + (p if axis == 1 else 0.0)], -1)


def source(c, x, y):
    """S = div F(U_exact): with it the manufactured fields are a steady solution of dU/dt = -div F + S."""
    h = 1e-30
    dFdx = np.imag(_flux(c, x + 1j * h, y + 0j, 0)) / h
    dGdy = np.imag(_flux(c, x + 0j, y + 1j * h, 1)) / h
    return dFdx + dGdy


def residual_norms(mesh, F, S):
    """RMS and max of F + S per component over the owned cells whose centroid lies in [1/3, 2/3]^2."""
    xc = mesh.cell_centroid
    sel = (mesh.cell_kind == L.CELL_OWNED) & np.all((xc[:, :2] >= 1.0 / 3.0) & (xc[:, :2] <= 2.0 / 3.0), axis=1)
    r = (F + S)[sel]
    return np.sqrt((r * r).mean(0)), np.abs(r).max(0)


def slopes(hs, norms):
    """Least-squares slope of log10(norm) against log10(h), per component."""
    lh = np.log10(np.asarray(hs))
    return np.array([np.polyfit(lh, np.log10(np.asarray(norms)[:, b]), 1)[0] for b in range(np.asarray(norms).shape[1])])


# the reference's inviscid parameter sets: (name, constants, flux calculator, PetscFV type, limiter,
# initial cells per direction, expected L2 orders, expected Linf orders); tolerance 0.2 as there. The
# least-squares cases run PETSc's default limiter (sin): with no limiter the orders come out near 2.
CASES = [
    ("low speed average", LOW, "avg", "upwind", "none", 4, [2, 2, 2, 2], [1.9, 1.8, 1.8, 1.8]),
    ("high speed average", HIGH, "avg", "upwind", "none", 4, [2, 2, 2, 2], [1.9, 1.8, 1.8, 1.8]),
    ("low speed ausm", LOW, "ausm", "upwind", "none", 16, [1.0, 1.0, 1.4, 1.0], [1.0, 1.0, 1.4, 1.0]),
    ("high speed ausm", HIGH, "ausm", "upwind", "none", 16, [1.0, 1.0, 1.0, 1.0], [1.0, 1.0, 1.0, 1.0]),
    ("low speed ausmpup", LOW, "ausmpup", "upwind", "none", 16, [1.0, 1.0, 1.2, 1.0], [1.0, 1.0, 1.2, 1.0]),
    ("high speed ausmpup", HIGH, "ausmpup", "upwind", "none", 16, [1.0, 1.0, 1.0, 1.0], [1.0, 1.0, 1.0, 1.0]),
    ("low speed ausm leastsquares", LOW, "ausm", "leastsquares", "sin", 16, [1.5, 1.5, 1.5, 1.5], [1.0, 1.0, 1.0, 1.0]),
    ("high speed ausm leastsquares", HIGH, "ausm", "leastsquares", "sin", 16, [1.5, 1.5, 1.5, 1.5], [1.0, 0.5, 1.0, 1.0]),
]
LEVELS = 4


def workload(case, level):
    """Mesh, conserved state (exact at every centroid, ghosts included: the reference's ghost function
    evaluates the exact solution half a cell beyond the face) and source of one refinement level."""
    from ablate_b200 import fv
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    name, c, flux, recon, lim, n0, _, _ = case
    n = n0 * 2 ** level
    mesh = box_mesh((n, n), order="morton")
    xc = mesh.cell_centroid
    U = conserved(c, xc[:, 0], xc[:, 1])
    S = source(c, xc[:, 0], xc[:, 1])
    eos = fv.PerfectGas({"gamma": GAMMA, "Rgas": 287.0})
    fc = {"avg": fv.AverageFlux(), "ausm": fv.Ausm(), "ausmpup": fv.AusmpUp(0.3)}[flux]
    w = Workload("mms", mesh, eos, [fv.NavierStokesTransport({}, eos, fc)], recon, lim, U, name)
    return w, S, 1.0 / n
