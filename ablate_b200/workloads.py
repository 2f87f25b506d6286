"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset is involved: every mesh and initial state is generated here from a fixed seed. Meshes
are numbered along a Morton curve by default (the order a DMPlexPermute with a space-filling-curve
ordering gives at setup); ``order="natural"`` gives DMPlexCreateBoxMesh's x-fastest numbering.

* ``sod2d``   2D Euler, perfect gas (gamma 1.4, R 287), n x n quads on [0,1]^2 with outflow ghost
              cells; Sod jump at x = 0.5 (rho 1 / 0.125, p 1e5 / 1e4, u = 0) times seeded Gaussian
              density bumps (amplitude 1 %, sigma 0.05). AUSM, first order.
* ``tgv3d``   3D compressible Navier-Stokes, perfect gas, n^3 periodic unit cube; Taylor-Green
              vortex at Mach 0.3 (T0 300 K, p0 101325 Pa, isothermal density) plus 0.5 % seeded white
              noise on the velocity. AUSM+up (mInf 0.3), least squares + minmod, constant
              mu = 1.8e-5 with k = mu cp / Pr (Pr 0.72).
* ``shear3d`` 3D Euler + species transport, n^3 hex box periodic in x and z with outflow ghosts in
              y, NASA-7 mixture of ``ns`` seeded species (cp/R in 2.5-6 over 300-3000 K); tanh shear
              layer with velocity ratio 3 plus seeded mass-fraction perturbations. AUSM+up,
              least squares + minmod.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import fv
from .mesh import Mesh, box_mesh, delaunay_mesh, ghost_interior_map


@dataclass
class Workload:
    name: str
    mesh: Mesh
    eos: object
    processes: list
    petscfv_type: str
    limiter: str
    U: np.ndarray  # (n_cells, nc) including ghost cells
    description: str
    boundary: tuple | None = None    # (condition table, per-cell condition index) for SetBoundary
    functional: tuple | None = None  # (cells, weights) of the wall-pressure functional

    def solver(self, device: int = 0) -> fv.FiniteVolumeSolver:
        return fv.FiniteVolumeSolver(self.mesh, self.eos, self.processes, self.petscfv_type, self.limiter, device=device)

    def physics(self):
        return fv.make_physics(self.eos, self.processes, self.petscfv_type, self.limiter)


def fill_outflow_ghosts(mesh: Mesh, U: np.ndarray) -> None:
    """Zero-gradient (outflow) ghost values: every ghost cell copies the interior cell across its face."""
    g = np.nonzero(mesh.cell_kind == L.CELL_BOUNDARY)[0]
    if g.size:
        U[g] = U[ghost_interior_map(mesh)]


def sod2d(n: int = 256, seed: int = 20261203, order: str = "morton") -> Workload:
    mesh = box_mesh((n, n), order=order)
    rng = np.random.default_rng(seed)
    gamma, R = 1.4, 287.0
    x = mesh.cell_centroid[:, 0]
    y = mesh.cell_centroid[:, 1]
    rho = np.where(x < 0.5, 1.0, 0.125)
    p = np.where(x < 0.5, 1e5, 1e4)
    bumps = np.zeros_like(x)
    for _ in range(8):
        cx, cy = rng.uniform(0.1, 0.9, 2)
        amp = rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 1.0)
        bumps += amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 0.05 ** 2))
    rho = rho * (1.0 + 0.01 * bumps)
    U = np.zeros((mesh.n_cells, 4))
    U[:, 0] = rho
    U[:, 1] = p / (gamma - 1.0)
    fill_outflow_ghosts(mesh, U)
    eos = fv.PerfectGas({"gamma": gamma, "Rgas": R})
    procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, fv.Ausm())]
    return Workload("sod2d", mesh, eos, procs, "upwind", "none", U,
                    f"2D Euler {n}x{n} quads, outflow ghosts, Sod + 1% Gaussian density bumps, AUSM, first order, FP64")


def tgv_state(mesh: Mesh, gamma=1.4, R=287.0, mach=0.3, T0=300.0, p0=101325.0, noise=0.005, seed=20261204):
    rng = np.random.default_rng(seed)
    a0 = np.sqrt(gamma * R * T0)
    V0 = mach * a0
    rho0 = p0 / (R * T0)
    k = 2.0 * np.pi
    x, y, z = (mesh.cell_centroid[:, d] for d in range(3))
    u = V0 * np.sin(k * x) * np.cos(k * y) * np.cos(k * z)
    v = -V0 * np.cos(k * x) * np.sin(k * y) * np.cos(k * z)
    w = np.zeros_like(u)
    p = p0 + rho0 * V0 ** 2 / 16.0 * (np.cos(2 * k * x) + np.cos(2 * k * y)) * (np.cos(2 * k * z) + 2.0)
    rho = p / (R * T0)
    vel = np.stack([u, v, w], 1) + noise * V0 * rng.standard_normal((mesh.n_cells, 3))
    U = np.zeros((mesh.n_cells, 5))
    U[:, 0] = rho
    U[:, 2:5] = rho[:, None] * vel
    U[:, 1] = p / (gamma - 1.0) + 0.5 * rho * (vel ** 2).sum(1)
    return U


def tgv3d(n: int = 128, seed: int = 20261204, order: str = "morton") -> Workload:
    mesh = box_mesh((n, n, n), periodic=(True, True, True), order=order)
    gamma, R = 1.4, 287.0
    U = tgv_state(mesh, gamma, R, seed=seed)
    mu, pr = 1.8e-5, 0.72
    cp = gamma * R / (gamma - 1.0)
    eos = fv.PerfectGas({"gamma": gamma, "Rgas": R})
    procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, fv.AusmpUp(0.3), fv.Constant(k=mu * cp / pr, mu=mu))]
    return Workload("tgv3d", mesh, eos, procs, "leastsquares", "minmod", U,
                    f"3D NS {n}^3 periodic hex, Taylor-Green M0.3 + 0.5% noise, AUSM+up + LSQ + minmod, mu 1.8e-5, Pr 0.72")


def tgv3d_slab(n: int, nparts: int, rank: int, seed: int = 20261204, order: str = "morton"):
    """Rank `rank`'s slab of the Taylor-Green case on an (n * nparts) x n x n periodic box, n^3 owned
    cells per rank with a two-layer halo (weak scaling); returns (LocalDomain, Workload)."""
    from .distributed import slab_domain
    dom = slab_domain((n * nparts, n, n), nparts, rank, order=order)
    w = tgv3d(2, seed)  # the physics of the case (its small mesh is replaced below)
    U = tgv_state(dom.mesh, seed=seed + rank)
    return dom, Workload("tgv3d", dom.mesh, w.eos, w.processes, w.petscfv_type, w.limiter, U,
                         f"3D NS {n}^3 cells per GPU of a periodic {n * nparts}x{n}x{n} hex box cut in x-slabs, Taylor-Green M0.3 + 0.5% "
                         "noise, AUSM+up + LSQ + minmod, mu 1.8e-5, Pr 0.72; 2-layer halo exchanged before every RHS")


def synthetic_nasa7(ns: int, seed: int) -> list[dict]:
    """Seeded NASA-7 species with cp/R rising from [2.5, 4] at 300 K to at most 6 at 3000 K, one
    polynomial on both ranges (T_mid 1000 K), formation enthalpy h_f/R in [-3e4, 1e4] K and molar
    mass in [2, 44] kg/kmol."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(ns):
        c300 = rng.uniform(2.5, 4.0)
        c3000 = rng.uniform(max(c300, 4.0), 6.0)
        # cp/R = a1 + a2 T + a3 T^2 through (300, c300) and (3000, c3000), concave (a3 <= 0)
        a3 = -rng.uniform(0.0, 0.15) * (c3000 - c300) / (2700.0 ** 2)
        a2 = ((c3000 - c300) - a3 * (3000.0 ** 2 - 300.0 ** 2)) / 2700.0
        a1 = c300 - a2 * 300.0 - a3 * 300.0 ** 2
        hf = rng.uniform(-3e4, 1e4)
        t = 298.15
        a6 = hf - (a1 * t + a2 / 2 * t ** 2 + a3 / 3 * t ** 3)
        a7 = rng.uniform(-10, 10)
        coeffs = [a1, a2, a3, 0.0, 0.0, a6, a7]
        mw = rng.uniform(2.0, 44.0)
        out.append({"name": f"S{k}", "composition": {"X": 1}, "T_ranges": [300.0, 1000.0, 3000.0], "low": coeffs, "high": coeffs,
                    "mw": mw})
    return out


def synthetic_mixture(ns: int, seed: int) -> fv.TChem:
    sp = synthetic_nasa7(ns, seed)
    eos = fv.TChem(sp, atomic_weights={"X": 1.0})
    eos.mw = np.array([s["mw"] for s in sp])
    return eos


def mixture_state(eos: fv.TChem, rho, vel, T, Y):
    """Conserved state from (rho, velocity, T, Y) with the NASA-7 sensible energy e_s(T)."""
    Ru = 8314.46261815324
    ns = Y.shape[1]
    Tref = 298.15

    def h_molar(k, TT):
        c = eos.nasa7[k]
        a = np.where((TT < c[0])[:, None], c[1:8][None, :], c[8:15][None, :])
        return Ru * TT * (a[:, 0] + TT * (a[:, 1] / 2 + TT * (a[:, 2] / 3 + TT * (a[:, 3] / 4 + TT * a[:, 4] / 5))) + a[:, 5] / TT)

    e = np.zeros_like(T)
    for k in range(ns):
        href = h_molar(k, np.array([Tref]))[0] / eos.mw[k]
        e += Y[:, k] * (h_molar(k, T) / eos.mw[k] - href - Ru * T / eos.mw[k])
    dim = vel.shape[1]
    U = np.zeros((rho.size, 2 + dim + ns))
    U[:, 0] = rho
    U[:, 2:2 + dim] = rho[:, None] * vel
    U[:, 1] = rho * (e + 0.5 * (vel ** 2).sum(1))
    U[:, 2 + dim:] = rho[:, None] * Y
    return U


def shear3d(n: int = 256, ns: int = 5, seed: int = 20261205, diffusion: bool = False, order: str = "morton") -> Workload:
    mesh = box_mesh((n, n, n), periodic=(True, False, True), order=order)
    rng = np.random.default_rng(seed)
    eos = synthetic_mixture(ns, seed + 1)
    x, y, z = (mesh.cell_centroid[:, d] for d in range(3))
    U1, U2, delta = 50.0, 150.0, 0.02
    ux = U1 + 0.5 * (U2 - U1) * (1.0 + np.tanh((y - 0.5) / delta))
    vel = np.stack([ux, 0.5 * np.sin(2 * np.pi * x) * np.exp(-((y - 0.5) / (4 * delta)) ** 2), np.zeros_like(ux)], 1)
    T = 300.0 + 600.0 * 0.5 * (1.0 + np.tanh((y - 0.5) / delta))
    Y = np.zeros((mesh.n_cells, ns))
    Y[:, 0] = 0.5 * (1.0 - np.tanh((y - 0.5) / delta))
    Y[:, 1] = 1.0 - Y[:, 0]
    Y += 0.02 * rng.uniform(0.0, 1.0, (mesh.n_cells, ns))
    Y /= Y.sum(1, keepdims=True)
    p = 101325.0
    Ru = 8314.46261815324
    W = 1.0 / (Y / eos.mw[None, :]).sum(1)
    rho = p * W / (Ru * T)
    U = mixture_state(eos, rho, vel, T, Y)
    fill_outflow_ghosts(mesh, U)
    flux = fv.AusmpUp(0.3)
    procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, flux), fv.SpeciesTransport(eos, flux)]
    if diffusion:
        procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, flux, fv.ConstantLewis(1.8e-5, 0.72, 1.0)),
                 fv.SpeciesTransport(eos, flux, fv.ConstantLewis(1.8e-5, 0.72, 1.0))]
    return Workload("shear3d", mesh, eos, procs, "leastsquares", "minmod", U,
                    f"3D Euler + {ns} species {n}^3 hex, NASA-7 mixture, tanh shear layer (ratio 3), AUSM+up + LSQ + minmod")


def channel_tets(n: int = 2_000_000, ns: int = 9, seed: int = 20261205) -> Workload:
    """Reacting-flow transport without chemistry on a seeded Delaunay tetrahedral mesh of the
    1 x 0.2 x 0.2 channel (about n cells): ns species with seeded NASA-7 data (cp/R in 2.5-6 over
    300-3000 K), mass fractions from layered profiles mixed with a seeded Dirichlet draw, T in
    300-2500 K (a hot core with 2 % seeded noise), p = 1 atm, a seeded velocity field; AUSM+up, least
    squares + van Leer, constant Lewis number 1 diffusion."""
    from .mesh import delaunay_mesh
    mesh = delaunay_mesh(n, seed=seed)
    rng = np.random.default_rng(seed)
    eos = synthetic_mixture(ns, seed)
    nc = mesh.n_cells
    x = mesh.cell_centroid
    # a hot core and layered composition with seeded cell-to-cell noise: T spans 300-2500 K
    r2 = ((x[:, 1] - 0.1) ** 2 + (x[:, 2] - 0.1) ** 2) / 0.01
    T = 300.0 + 2200.0 * np.exp(-2.0 * r2) * (0.6 + 0.4 * np.sin(2 * np.pi * x[:, 0])) ** 2
    T *= 1.0 + 0.02 * rng.standard_normal(nc)
    T = np.clip(T, 300.0, 2500.0)
    Ylayer = np.stack([1.0 + np.cos(2 * np.pi * (k + 1) * x[:, 0] + k) for k in range(ns)], 1) + 0.2
    Y = 0.8 * Ylayer / Ylayer.sum(1, keepdims=True) + 0.2 * rng.dirichlet(np.ones(ns) * 2.0, nc)
    W = 1.0 / (Y / eos.mw).sum(1)
    rho = 101325.0 * W / (8314.46261815324 * T)
    vel = np.stack([30.0 * np.sin(2 * np.pi * x[:, 1] / 0.2), 10.0 * np.cos(2 * np.pi * x[:, 0]), 5.0 * np.ones(nc)], 1)
    vel += 2.0 * rng.standard_normal((nc, 3))
    U = mixture_state(eos, rho, vel, T, Y)
    flux = fv.AusmpUp(0.3)
    tr = fv.ConstantLewis(1.8e-5, 0.72, 1.0)
    procs = [fv.NavierStokesTransport({}, eos, flux, tr), fv.SpeciesTransport(eos, flux, tr)]
    return Workload("channel_tets", mesh, eos, procs, "leastsquares", "vanleer", U,
                    f"3D {mesh.n_interior} seeded Delaunay tets in a 1x0.2x0.2 channel, {ns} NASA-7 species, AUSM+up + LSQ + van Leer, Le = 1")


def wall3d(n: int = 128, seed: int = 20261206, speed_mach: float = 0.3, order: str = "morton") -> Workload:
    """Wall-bounded variant of the Taylor-Green physics for the functional gradient: n^3 hex cells on
    the unit cube, periodic in z, a Dirichlet inlet at x = 0 (uniform flow at Mach `speed_mach` along
    x, T 300 K, p 101325 Pa), outflow at x = 1, no-slip walls at y = 0 and y = 1. Initial state: the
    inlet flow with 0.5 % seeded white noise on the velocity and on the density. The functional is the
    pressure integrated over the wall patch y = 0, 0 < x < 0.25 next to the inlet (the cells next to
    those wall faces, weighted by the face area), which the inlet reaches within a few steps. AUSM+up + least squares + minmod, constant mu = 1.8e-5, Pr 0.72."""
    from .adjoint import inlet_state
    mesh = box_mesh((n, n, n), periodic=(False, False, True), order=order)
    rng = np.random.default_rng(seed)
    gamma, R, T0, p0 = 1.4, 287.0, 300.0, 101325.0
    rho0 = p0 / (R * T0)
    V = speed_mach * np.sqrt(gamma * R * T0)
    nc = mesh.n_cells
    rho = rho0 * (1.0 + 0.005 * rng.standard_normal(nc))
    vel = np.zeros((nc, 3))
    vel[:, 0] = V
    vel += 0.005 * V * rng.standard_normal((nc, 3))
    U = np.zeros((nc, 5))
    U[:, 0] = rho
    U[:, 2:5] = rho[:, None] * vel
    U[:, 1] = p0 / (gamma - 1.0) + 0.5 * rho * (vel ** 2).sum(1)
    inlet, _ = inlet_state(rho0, p0, V, (1.0, 0.0, 0.0), gamma)
    table = [(L.BC_DIRICHLET, list(inlet), False), (L.BC_OUTFLOW, None, False), (L.BC_NOSLIP_WALL, None, False)]
    cell_bc = np.zeros(nc, np.int32)
    ghosts = np.nonzero(mesh.cell_kind == L.CELL_BOUNDARY)[0]
    gx, gy = mesh.cell_centroid[ghosts, 0], mesh.cell_centroid[ghosts, 1]
    cell_bc[ghosts] = np.where(gx < 0.0, 0, np.where(gx > 1.0, 1, 2))
    inner = ghost_interior_map(mesh)
    patch = (gy < 0.0) & (gx > 0.0) & (gx < 0.25)
    area = 1.0 / n ** 2
    fill_outflow_ghosts(mesh, U)
    mu, pr = 1.8e-5, 0.72
    cp = gamma * R / (gamma - 1.0)
    eos = fv.PerfectGas({"gamma": gamma, "Rgas": R})
    procs = [fv.NavierStokesTransport({"cfl": 0.5}, eos, fv.AusmpUp(0.3), fv.Constant(k=mu * cp / pr, mu=mu))]
    return Workload("wall3d", mesh, eos, procs, "leastsquares", "minmod", U,
                    f"3D NS {n}^3 hex channel: Dirichlet inlet M{speed_mach} at x=0, outflow x=1, no-slip walls y=0,1, periodic z; "
                    "AUSM+up + LSQ + minmod, mu 1.8e-5, Pr 0.72; functional: pressure integrated over the wall patch y=0, 0<x<0.25",
                    boundary=(table, cell_bc), functional=(inner[patch], np.full(int(patch.sum()), area)))


def initial_aux(w: Workload) -> np.ndarray:
    """Aux array with a 300 K temperature guess (what an ABLATE aux vector holds before its first update)."""
    dim = w.mesh.dim
    ns = len(w.eos.GetSpeciesVariables())
    a = np.zeros((w.mesh.n_cells, 1 + dim + ns))
    a[:, 0] = 300.0
    return a
