"""Small seeded RHS cases shared by the parity tests (each finishes in well under a second on the oracle)."""
from __future__ import annotations

import zlib

import numpy as np

from ablate_b200 import _lib as L
from ablate_b200 import fv, workloads
from ablate_b200.mesh import box_mesh
from ablate_b200.workloads import Workload, fill_outflow_ghosts, mixture_state, synthetic_mixture


def _perturbed_state(mesh, rng, dim, ns=0, eos=None):
    n = mesh.n_cells
    x = mesh.cell_centroid
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.05 * rng.standard_normal(n)
    vel = 40.0 * rng.standard_normal((n, dim)) + 80.0
    if eos is None:
        p = 1e5 * (1.0 + 0.2 * np.cos(2 * np.pi * x[:, 0])) * (1.0 + 0.05 * rng.standard_normal(n))
        U = np.zeros((n, 2 + dim + ns))
        U[:, 0] = rho
        U[:, 2:2 + dim] = rho[:, None] * vel
        U[:, 1] = p / 0.4 + 0.5 * rho * (vel ** 2).sum(1)
        if ns:
            Y = rng.dirichlet(np.ones(ns), n)
            U[:, 2 + dim:] = rho[:, None] * Y
        return U
    T = 600.0 + 300.0 * np.sin(2 * np.pi * x[:, 1]) + 20.0 * rng.standard_normal(n)
    Y = rng.dirichlet(np.ones(ns) * 2.0, n)
    return mixture_state(eos, rho, vel, T, Y)


def case(name: str) -> Workload:
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "sod2d_ausm_upwind":
        return workloads.sod2d(16)
    if name == "tgv3d_ausmpup_lsq_minmod_visc":
        return workloads.tgv3d(8)
    if name == "tgv3d_mixed_check":
        return workloads.tgv3d(16)
    if name == "tgv3d_natural_order":
        return workloads.tgv3d(8, order="natural")
    if name == "sod2d_natural_order":
        return workloads.sod2d(16, order="natural")
    if name.startswith("box2d_"):
        # 2D with ghost boundaries, LSQ, the limiter/flux named in the case
        _, flux, lim, tr = name.split("_")
        mesh = box_mesh((12, 9), lower=(0, 0), upper=(1.2, 0.9), periodic=(False, True))
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0})
        fc = {"ausm": fv.Ausm(), "ausmpup": fv.AusmpUp(0.3), "riemann": fv.Riemann(eos), "avg": fv.AverageFlux(), "off": fv.OffFlux()}[flux]
        trm = {"none": None, "const": fv.Constant(k=0.025, mu=1.8e-5), "suth": fv.Sutherland(eos)}[tr]
        U = _perturbed_state(mesh, rng, 2)
        U[mesh.cell_kind == L.CELL_BOUNDARY] *= 1.0 + 0.01 * rng.standard_normal((int((mesh.cell_kind == L.CELL_BOUNDARY).sum()), 4))
        return Workload(name, mesh, eos, [fv.NavierStokesTransport({}, eos, fc, trm)], "leastsquares" if lim != "upwind" else "upwind",
                        lim if lim != "upwind" else "none", U, name)
    if name.startswith("box1d_visc"):
        # 1D Navier-Stokes with conduction and viscosity, LSQ + minmod: the 1D face stencil
        periodic = name.endswith("_periodic")
        mesh = box_mesh((32,), periodic=(periodic,))
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0})
        U = _perturbed_state(mesh, rng, 1)
        procs = [fv.NavierStokesTransport({}, eos, fv.AusmpUp(0.3), fv.Constant(k=0.6, mu=2e-3))]
        return Workload(name, mesh, eos, procs, "leastsquares", "minmod", U, name)
    if name == "box1d_riemann_upwind":
        mesh = box_mesh((40,))
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0})
        x = mesh.cell_centroid[:, 0]
        U = np.zeros((mesh.n_cells, 3))
        U[:, 0] = np.where(x < 0.5, 1.0, 0.125)
        U[:, 1] = np.where(x < 0.5, 1e5, 1e4) / 0.4
        fill_outflow_ghosts(mesh, U)
        return Workload(name, mesh, eos, [fv.NavierStokesTransport({}, eos, fv.Riemann(eos))], "upwind", "none", U, name)
    if name.startswith("species3d_"):
        ns = int(name.split("_")[1][2:])
        mesh = box_mesh((6, 5, 4), lower=(0, 0, 0), upper=(0.6, 0.5, 0.4), periodic=(True, False, False))
        eos = synthetic_mixture(ns, 7)
        U = _perturbed_state(mesh, rng, 3, ns, eos)
        flux = fv.AusmpUp(0.3)
        if name.endswith("_dk"):
            # the Constant model with one diffusivity per species (the VariableDiffusionCoefficient fluxes)
            tr = fv.Constant(k=0.03, mu=2e-5, diff=np.linspace(2e-5, 1.2e-4, ns))
        else:
            tr = fv.ConstantLewis(1.8e-5, 0.72, 1.0)
        procs = [fv.NavierStokesTransport({}, eos, flux, tr), fv.SpeciesTransport(eos, flux, tr)]
        return Workload(name, mesh, eos, procs, "leastsquares", "vanleer", U, name)
    if name == "gri30_box3d":
        # the reference's 53-species gri30 thermodynamics (the input of its tChemTests.cpp) on a small
        # box: a count without an instance of its own, run padded in the largest species instance
        from tests import golden_cases as G
        mesh = box_mesh((5, 4, 3), lower=(0, 0, 0), upper=(0.5, 0.4, 0.3), periodic=(True, False, False))
        eos = G.gri30_eos()
        U = _perturbed_state(mesh, rng, 3, len(eos.GetSpeciesVariables()), eos)
        flux = fv.AusmpUp(0.3)
        tr = fv.ConstantLewis(1.8e-5, 0.72, 1.0)
        procs = [fv.NavierStokesTransport({}, eos, flux, tr), fv.SpeciesTransport(eos, flux, tr)]
        return Workload(name, mesh, eos, procs, "leastsquares", "minmod", U, name)
    if name == "compact3d_avg_ns5":
        # the compact NS + species process with the average flux (no direction: the averaged species
        # advection), per-species diffusivities
        mesh = box_mesh((6, 5, 4), lower=(0, 0, 0), upper=(0.6, 0.5, 0.4), periodic=(True, False, False))
        eos = synthetic_mixture(5, 7)
        U = _perturbed_state(mesh, rng, 3, 5, eos)
        tr = fv.Constant(k=0.03, mu=2e-5, diff=np.linspace(3e-5, 9e-5, 5))
        procs = [fv.CompactCompressibleNSSpeciesTransport({}, eos, fv.AverageFlux(), tr)]
        return Workload(name, mesh, eos, procs, "leastsquares", "minmod", U, name)
    if name.startswith("pgspecies3d_"):
        ns = int(name.split("_")[1][2:])
        mesh = box_mesh((5, 4, 4), periodic=(False, True, True))
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0}, [f"S{k}" for k in range(ns)])
        U = _perturbed_state(mesh, rng, 3, ns)
        flux = fv.Ausm()
        tr = fv.Constant(k=0.03, mu=2e-5, diff=1e-4)
        procs = [fv.NavierStokesTransport({}, eos, flux, tr), fv.SpeciesTransport(eos, flux, tr)]
        return Workload(name, mesh, eos, procs, "leastsquares", "minmod", U, name)
    if name == "shear3d_ns5":
        # the 256^3 five-species shear layer's generator (outflow ghosts in y, NASA-7, AUSM+up, LSQ +
        # minmod) at 16^3, large enough for its record tables (7 cone-weight and 4 geometry classes)
        return workloads.shear3d(16, 5)
    if name == "walled_channel3d":
        # the walled channel of the derivative studies (inlet, outflow, no-slip walls, periodic z)
        return workloads.wall3d(10)
    if name.startswith("tets3d_"):
        # seeded Delaunay tets of the 1 x 0.2 x 0.2 channel: variable cone sizes, ghosts on every side
        if name == "tets3d_ns9":
            return workloads.channel_tets(1500, 9, seed=zlib.crc32(name.encode()))
        mesh = workloads.delaunay_mesh(1200, seed=zlib.crc32(name.encode()))
        eos = fv.PerfectGas({"gamma": 1.4, "Rgas": 287.0})
        U = _perturbed_state(mesh, rng, 3)
        procs = [fv.NavierStokesTransport({}, eos, fv.Ausm(), fv.Constant(k=0.03, mu=2e-5))]
        return Workload(name, mesh, eos, procs, "leastsquares", "minmod", U, name)
    raise KeyError(name)


CASES = [
    "sod2d_ausm_upwind",
    "sod2d_natural_order",
    "tgv3d_natural_order",
    "box1d_riemann_upwind",
    "box1d_visc",
    "box1d_visc_periodic",
    "tgv3d_ausmpup_lsq_minmod_visc",
    "box2d_ausm_upwind_none",
    "box2d_ausm_minmod_const",
    "box2d_ausmpup_vanleer_suth",
    "box2d_riemann_vanalbada_none",
    "box2d_avg_sin_const",
    "box2d_off_zero_const",
    "box2d_ausm_none_none",
    "species3d_ns5",
    "species3d_ns9",
    "species3d_ns5_dk",
    "compact3d_avg_ns5",
    "pgspecies3d_ns2",
    "tets3d_ns9",
    "tets3d_pg_minmod",
    "shear3d_ns5",
    "walled_channel3d",
]


def block_errors(F_test: np.ndarray, F_ref: np.ndarray, owned: np.ndarray, neuler: int) -> dict:
    """Norm-wise relative error ||dF||_2 / ||F||_2 per field block over owned cells."""
    out = {}
    blocks = {"euler": slice(0, neuler)}
    if F_ref.shape[1] > neuler:
        blocks["densityYi"] = slice(neuler, F_ref.shape[1])
    for name, sl in blocks.items():
        a = F_test[owned, sl]
        b = F_ref[owned, sl]
        den = np.linalg.norm(b)
        out[name] = float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))
    return out
