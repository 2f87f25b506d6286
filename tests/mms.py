"""Manufactured solutions of the reference's RHS convergence test (compressibleFlowMmsSourceTests.cpp):
smooth 2D Euler fields built from sines and cosines, the source that makes them steady, and the
convergence orders of the residual RHS(U_exact) + S over the central third of the unit square.

The source is the divergence of the exact Euler flux, formed here by complex-step differentiation
(f'(x) = Im f(x + ih) / h, exact to rounding) of the flux of the manufactured fields, rather than from
a closed form; for the conduction and viscous sets it adds the divergence of the exact diffusive flux.
"""
from __future__ import annotations

import numpy as np

from ablate_b200 import _lib as L

# the reference's 2D parameter sets: field -> (phi0, phiX, phiY, phiZ, aPhiX, aPhiY, aPhiZ); gamma 1.4,
# R 287, L 1; the 2D sets carry no z terms and no w field
LOW = {"rho": (1.0, 0.15, -0.1, 0.0, 1.0, 0.5, 0.0), "u": (70.0, 5.0, -7.0, 0.0, 1.5, 0.6, 0.0),
       "v": (90.0, -15.0, -8.5, 0.0, 0.5, 2.0 / 3.0, 0.0), "p": (1e5, 0.2e5, 0.5e5, 0.0, 2.0, 1.0, 0.0)}
HIGH = {"rho": (1.0, 0.15, -0.1, 0.0, 1.0, 0.5, 0.0), "u": (800.0, 50.0, -30.0, 0.0, 1.5, 0.6, 0.0),
        "v": (800.0, -75.0, 40.0, 0.0, 0.5, 2.0 / 3.0, 0.0), "p": (1e5, 0.2e5, 0.5e5, 0.0, 2.0, 1.0, 0.0)}
# the reference's 3D set (low speed)
LOW3D = {"rho": (1.0, 0.15, -0.1, 0.0, 1.0, 0.5, 0.4), "u": (70.0, 5.0, -7.0, 5.0, 1.5, 0.6, 0.5),
         "v": (90.0, -15.0, -8.5, 6.5, 0.5, 2.0 / 3.0, 0.6), "w": (80.0, -25.0, 8.2, -10.0, 0.75, 0.2, 0.7),
         "p": (1e5, 0.2e5, 0.5e5, 0.4e5, 2.0, 1.0, 0.8)}
GAMMA = 1.4
R_GAS = 287.0


def primitives(c, X):
    """rho, the velocity components and p at the points X = (x, y[, z]) (arrays, real or complex).
    Which term carries a sine and which a cosine follows the reference:
    rho = r0 + rY cos + rX sin + rZ sin, u = u0 + uY cos + uZ cos + uX sin,
    v = v0 + vX cos + vY sin + vZ sin, w = w0 + wZ cos + wX sin + wY sin, p = p0 + pX cos + pZ cos + pY sin."""
    pi = np.pi
    x, y = X[0], X[1]
    z = X[2] if len(X) > 2 else 0.0 * x

    def field(name, cos_axes):
        f0, fx, fy, fz, ax, ay, az = c[name]
        out = f0 + 0.0 * x
        for amp, a, t, cs in ((fx, ax, x, "x" in cos_axes), (fy, ay, y, "y" in cos_axes), (fz, az, z, "z" in cos_axes)):
            out = out + amp * (np.cos(a * pi * t) if cs else np.sin(a * pi * t))
        return out

    rho = field("rho", "y")
    vel = [field("u", "yz"), field("v", "x")] + ([field("w", "z")] if len(X) > 2 else [])
    p = field("p", "xz")
    return rho, vel, p


def conserved(c, X):
    rho, vel, p = primitives(c, X)
    E = p / ((GAMMA - 1.0) * rho) + 0.5 * sum(v * v for v in vel)
    return np.stack([rho, rho * E] + [rho * v for v in vel], -1)


def _flux(c, X, axis):
    """The Euler flux through a face of unit normal e_axis."""
    rho, vel, p = primitives(c, X)
    E = p / ((GAMMA - 1.0) * rho) + 0.5 * sum(v * v for v in vel)
    un = vel[axis]
    return np.stack([rho * un, (rho * E + p) * un] + [rho * v * un + (p if b == axis else 0.0) for b, v in enumerate(vel)], -1)


def _shift(X, axis, d):
    return tuple(t + d if b == axis else t + 0.0 * d for b, t in enumerate(X))


def _grad(fn, X):
    """The gradient of a real function of the points X by complex steps."""
    h = 1e-30
    return [np.imag(fn(_shift(X, a, 1j * h))) / h for a in range(len(X))]


def _diffusive_flux(c, X, axis, mu, k):
    """NavierStokesTransport::DiffusionFlux through a face of unit normal e_axis: momentum -tau_(b,axis),
    energy -(sum_b u_b tau_(axis,b) + k dT/dx_axis), with tau = mu (grad u + grad u^T) - 2/3 mu div u I
    and T = p / (rho R)."""
    dim = len(X)
    rho, vel, p = primitives(c, X)
    du = [_grad(lambda Y, b=b: primitives(c, Y)[1][b], X) for b in range(dim)]  # du[b][a] = d u_b / d x_a
    dT = _grad(lambda Y: primitives(c, Y)[2] / (primitives(c, Y)[0] * R_GAS), X)
    div = sum(du[b][b] for b in range(dim))
    tau = [[mu * (du[b][a] + du[a][b]) - (2.0 / 3.0 * mu * div if a == b else 0.0) for b in range(dim)] for a in range(dim)]
    energy = -(sum(vel[b] * tau[axis][b] for b in range(dim)) + k * dT[axis])
    return np.stack([0.0 * rho, energy] + [-tau[b][axis] for b in range(dim)], -1)


def source(c, X, mu=0.0, k=0.0):
    """S = div (F + F_d)(U_exact), F the Euler flux and F_d the diffusive flux: with it the manufactured
    fields are a steady solution of dU/dt = -div (F + F_d) + S. The Euler part by complex steps; the
    diffusive part, which holds first derivatives already, by central differences of step 1e-5 of its
    complex-step form (error near 1e-10 of its size)."""
    h = 1e-30
    X = tuple(np.asarray(t, float) for t in X)
    S = sum(np.imag(_flux(c, _shift(X, a, 1j * h), a)) / h for a in range(len(X)))
    if mu or k:
        d = 1e-5
        for a in range(len(X)):
            S = S + (_diffusive_flux(c, _shift(X, a, d), a, mu, k) - _diffusive_flux(c, _shift(X, a, -d), a, mu, k)) / (2 * d)
    return S


def residual_norms(mesh, F, S):
    """RMS and max of F + S per component over the owned cells whose centroid lies in [1/3, 2/3]^dim."""
    xc = mesh.cell_centroid[:, :mesh.dim]
    sel = (mesh.cell_kind == L.CELL_OWNED) & np.all((xc >= 1.0 / 3.0) & (xc <= 2.0 / 3.0), axis=1)
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
# the parameter sets with conduction (k 1000) and with conduction and viscosity (mu 300): average
# flux, first order; (name, constants, dim, mu, k, initial cells, levels, expected L2, expected Linf)
VISCOUS_CASES = [
    ("low speed average with conduction", LOW, 2, 0.0, 1000.0, 4, 4, [2, 2, 2, 2], [1.9, 1.8, 1.8, 1.8]),
    ("high speed average with conduction", HIGH, 2, 0.0, 1000.0, 4, 4, [2, 2, 2, 2], [1.9, 1.8, 1.8, 1.8]),
    ("low speed average with conduction and diffusion", LOW, 2, 300.0, 1000.0, 4, 4, [2, 2, 2, 2.2], [1.9, 1.8, 1.8, 2.0]),
    ("high speed average with conduction and diffusion", HIGH, 2, 300.0, 1000.0, 4, 4, [2, 2, 2, 2.0], [1.9, 2.0, 1.8, 1.8]),
    ("low speed average with conduction and diffusion 3D", LOW3D, 3, 300.0, 1000.0, 10, 2,
     [2.1, 2.2, 2.2, 2.2, 2.0], [1.9, 2.2, 2.0, 2.2, 2.0]),
]
LEVELS = 4


def levels(case):
    return case[6] if len(case) == 9 else LEVELS


def workload(case, level):
    """Mesh, conserved state (exact at every centroid, ghosts included: the reference's ghost function
    evaluates the exact solution half a cell beyond the face) and source of one refinement level."""
    from ablate_b200 import fv
    from ablate_b200.mesh import box_mesh
    from ablate_b200.workloads import Workload
    eos = fv.PerfectGas({"gamma": GAMMA, "Rgas": R_GAS})
    if len(case) == 9:  # a viscous set
        name, c, dim, mu, k, n0 = case[:6]
        n = n0 * 2 ** level
        mesh = box_mesh((n,) * dim, order="morton")
        X = tuple(mesh.cell_centroid[:, a] for a in range(dim))
        procs = [fv.NavierStokesTransport({}, eos, fv.AverageFlux(), fv.Constant(k=k, mu=mu))]
        w = Workload("mms", mesh, eos, procs, "upwind", "none", conserved(c, X), name)
        return w, source(c, X, mu, k), 1.0 / n
    name, c, flux, recon, lim, n0 = case[:6]
    n = n0 * 2 ** level
    mesh = box_mesh((n, n), order="morton")
    X = (mesh.cell_centroid[:, 0], mesh.cell_centroid[:, 1])
    fc = {"avg": fv.AverageFlux(), "ausm": fv.Ausm(), "ausmpup": fv.AusmpUp(0.3)}[flux]
    w = Workload("mms", mesh, eos, [fv.NavierStokesTransport({}, eos, fc)], recon, lim, conserved(c, X), name)
    return w, source(c, X), 1.0 / n
