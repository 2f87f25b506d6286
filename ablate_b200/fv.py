"""Host-side mirror of ABLATE's FV process interfaces, driving the B200 backend through its C ABI.

The objects here carry the same names and constructor arguments as the reference classes they stand
for, and ``FiniteVolumeSolver`` wires them the way ``Process::Setup`` / ``RegisterRHSFunction`` do:

  eos.PerfectGas(parameters, species)              src/eos/perfectGas.cpp:4-7 (gamma 1.4, Rgas 287 defaults)
  eos.TChem(species thermo)                        src/eos/tChem.cpp (NASA-7 thermodynamics only)
  fluxCalculator.{Ausm, AusmpUp, Riemann, AverageFlux, OffFlux}
                                                   src/finiteVolume/fluxCalculator/*.cpp
  transport.{Constant, Sutherland, ConstantLewis}  src/eos/transport/{constant,sutherland}.cpp
  processes.{NavierStokesTransport, SpeciesTransport}
                                                   src/finiteVolume/processes/{navierStokesTransport,speciesTransport}.cpp
  FiniteVolumeSolver.ComputeRHSFunction            src/finiteVolume/finiteVolumeSolver.cpp:233-291

Every numeric path goes to the sm_100a kernels of ``lib/libablate_fv.so``; there is no CPU
implementation in this package.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L


# ---------------------------------------------------------------------------------------------
# eos
# ---------------------------------------------------------------------------------------------
class PerfectGas:
    """ablate::eos::PerfectGas (src/eos/perfectGas.cpp:4-7)."""

    def __init__(self, parameters: dict | None = None, species: Sequence[str] = ()):
        parameters = parameters or {}
        self.gamma = float(parameters.get("gamma", 1.4))
        self.rGas = float(parameters.get("Rgas", 287.0))
        self.species = list(species)

    def GetSpecificHeatRatio(self):
        return self.gamma

    def GetGasConstant(self):
        return self.rGas

    def GetSpeciesVariables(self):
        return list(self.species)

    def _fill(self, p: L.PhysicsDesc, keep: list):
        p.eos = L.EOS_PERFECT_GAS
        p.gamma = self.gamma
        p.r_gas = self.rGas


# atomic weights (kg/kmol) used to form species molar masses from their elemental composition
ATOMIC_WEIGHTS = {"H": 1.00797, "O": 15.9994, "C": 12.01115, "N": 14.0067, "AR": 39.948, "Ar": 39.948, "HE": 4.0026, "He": 4.0026}


class TChem:
    """NASA-7 mixture EOS (the thermodynamics of ablate::eos::TChem, src/eos/tChem.cpp).

    ``species`` is a list of dicts with keys name, composition (element -> count), T_ranges
    [T_low, T_mid, T_high], low (7 coefficients), high (7 coefficients), as in a Cantera YAML file.
    """

    def __init__(self, species: list[dict], atomic_weights: dict | None = None):
        aw = atomic_weights or ATOMIC_WEIGHTS
        self.names = [s["name"] for s in species]
        ns = len(species)
        self.nasa7 = np.zeros((ns, 15))
        self.mw = np.zeros(ns)
        for k, s in enumerate(species):
            self.nasa7[k, 0] = s["T_ranges"][1]
            self.nasa7[k, 1:8] = s["low"]
            self.nasa7[k, 8:15] = s["high"]
            self.mw[k] = sum(aw[el] * n for el, n in s["composition"].items())

    @classmethod
    def from_yaml(cls, path, atomic_weights: dict | None = None):
        """Read NASA-7 species from a Cantera-format YAML mechanism (YAML 1.1 booleans disabled so that
        species such as NO and elements such as N stay strings)."""
        import yaml

        class Loader(yaml.SafeLoader):
            pass

        Loader.yaml_implicit_resolvers = {k: [(t, r) for t, r in v if t != "tag:yaml.org,2002:bool"]
                                          for k, v in yaml.SafeLoader.yaml_implicit_resolvers.items()}
        doc = yaml.load(open(path).read(), Loader=Loader)
        species = []
        for sp in doc["species"]:
            th = sp["thermo"]
            species.append({"name": sp["name"], "composition": sp["composition"], "T_ranges": th["temperature-ranges"],
                            "low": th["data"][0], "high": th["data"][1]})
        return cls(species, atomic_weights)

    def GetSpeciesVariables(self):
        return list(self.names)

    def _fill(self, p: L.PhysicsDesc, keep: list):
        p.eos = L.EOS_NASA7
        a = np.ascontiguousarray(self.nasa7)
        m = np.ascontiguousarray(self.mw)
        keep += [a, m]
        p.nasa7 = L.dptr(a)
        p.mw = L.dptr(m)
        p.gamma = 1.4
        p.r_gas = 287.0


# ---------------------------------------------------------------------------------------------
# flux calculators
# ---------------------------------------------------------------------------------------------
class _Flux:
    kind = L.FLUX_OFF

    def _params(self):
        return 0.0, 1.0, 1.4

    def GetFluxCalculatorFunction(self):
        """Vectorised FluxCalculatorFunction evaluated on the device: (massFlux, p12, direction) arrays."""
        kind = self.kind
        minf, alpha, gamma = self._params()

        def fn(uL, aL, rhoL, pL, uR, aR, rhoR, pR):
            arrs = [np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64) for x in (uL, aL, rhoL, pL, uR, aR, rhoR, pR)]
            n = arrs[0].size
            mf, p12 = np.zeros(n), np.zeros(n)
            d = np.zeros(n, np.int32)
            L.check(L.lib.abl_flux_calculator_batch(kind, minf, alpha, gamma, n, *[L.dptr(a) for a in arrs], L.dptr(mf), L.dptr(p12),
                                                    L.iptr(d)), "flux calculator")
            return mf, p12, d

        return fn


class Ausm(_Flux):
    kind = L.FLUX_AUSM


class AusmpUp(_Flux):
    """AusmpUp(mInf, pgs): pgs may be a PressureGradientScaling-like object with GetAlpha() or a number."""
    kind = L.FLUX_AUSMPUP

    def __init__(self, mInf: float = 0.0, pgs=None):
        self.mInf = float(mInf)
        self.pgs = pgs

    def _alpha(self):
        if self.pgs is None:
            return 1.0
        return float(self.pgs.GetAlpha() if hasattr(self.pgs, "GetAlpha") else self.pgs)

    def _params(self):
        return self.mInf, self._alpha(), 1.4


class Riemann(_Flux):
    kind = L.FLUX_RIEMANN

    def __init__(self, eos):
        if not isinstance(eos, PerfectGas):
            raise ValueError("Riemann only accepts EOS of type eos::PerfectGas")
        self.gamma = eos.GetSpecificHeatRatio()

    def _params(self):
        return 0.0, 1.0, self.gamma


class AverageFlux(_Flux):
    kind = L.FLUX_AVERAGE


class OffFlux(_Flux):
    kind = L.FLUX_OFF


class PressureGradientScaling:
    """Only the alpha used by AusmpUp (src/finiteVolume/processes/pressureGradientScaling.hpp:84)."""

    def __init__(self, eos=None, alphaInit: float = 1.0, *args):
        self.alpha = float(alphaInit)

    def GetAlpha(self):
        return self.alpha


# ---------------------------------------------------------------------------------------------
# transport
# ---------------------------------------------------------------------------------------------
class Constant:
    """src/eos/transport/constant.cpp: constant k, mu and diffusivity; the diffusivity is one value, or
    one per species (then SpeciesTransport registers its VariableDiffusionCoefficient fluxes)."""

    def __init__(self, k: float = 0.0, mu: float = 0.0, diff=0.0):
        self.k, self.mu = float(k), float(mu)
        if np.ndim(diff) == 0:
            self.diff, self.species_diff = float(diff), None
        else:
            self.diff, self.species_diff = 0.0, np.ascontiguousarray(diff, dtype=np.float64)

    def _fill(self, p):
        p.transport = L.TRANSPORT_CONSTANT
        p.k, p.mu, p.diff = self.k, self.mu, self.diff
        if self.species_diff is not None:
            if len(self.species_diff) != p.n_species:
                raise ValueError("The diffusion property size must be 1 or number of species")
            p.species_diff = L.dptr(self.species_diff)


class Sutherland:
    def __init__(self, eos=None):
        self.eos = eos

    def _fill(self, p):
        p.transport = L.TRANSPORT_SUTHERLAND


class ConstantLewis:
    """Constant viscosity, k = mu cp / Pr, species diffusivity D = k / (rho cp Le). No reference counterpart."""

    def __init__(self, mu: float, prandtl: float = 0.72, lewis: float = 1.0):
        self.mu, self.prandtl, self.lewis = float(mu), float(prandtl), float(lewis)

    def _fill(self, p):
        p.transport = L.TRANSPORT_CONSTANT_LEWIS
        p.mu, p.k, p.diff = self.mu, self.prandtl, self.lewis


# ---------------------------------------------------------------------------------------------
# processes
# ---------------------------------------------------------------------------------------------
class NavierStokesTransport:
    """src/finiteVolume/processes/navierStokesTransport.cpp:10-97"""

    def __init__(self, parameters: dict | None, eos, fluxCalculator=None, transport=None, pgs=None):
        self.parameters = parameters or {}
        self.eos, self.fluxCalculator, self.transport = eos, fluxCalculator, transport

    def Setup(self, flow: "FiniteVolumeSolver"):
        if self.fluxCalculator is not None:
            flow.RegisterRHSFunction("NavierStokesTransport::AdvectionFlux", self.fluxCalculator)
        if self.transport is not None:
            flow.RegisterRHSFunction("NavierStokesTransport::DiffusionFlux", self.transport)


class SpeciesTransport:
    """src/finiteVolume/processes/speciesTransport.cpp:7-96"""

    def __init__(self, eos, fluxCalculator=None, transport=None, parameters: dict | None = None):
        self.eos, self.fluxCalculator, self.transport = eos, fluxCalculator, transport

    def Setup(self, flow: "FiniteVolumeSolver"):
        if not self.eos.GetSpeciesVariables():
            return
        if self.fluxCalculator is not None:
            flow.RegisterRHSFunction("SpeciesTransport::AdvectionFlux", self.fluxCalculator)
        if self.transport is not None:
            flow.RegisterRHSFunction("SpeciesTransport::DiffusionSpeciesFlux", self.transport)


class CompactCompressibleNSSpeciesTransport:
    """src/finiteVolume/processes/compactCompressibleNSSpeciesTransport.cpp:12-160: Navier-Stokes and
    species transport in one process. Its fluxes are NavierStokesTransport's and SpeciesTransport's,
    except the species advection where the flux calculator gives no direction (the average flux):
    there rho Y_k is carried as (rho Y_L + rho Y_R) / (rho_L + rho_R)."""

    def __init__(self, parameters: dict | None, eos, fluxCalculator=None, transport=None, pgs=None):
        self.parameters = parameters or {}
        self.eos, self.fluxCalculator, self.transport = eos, fluxCalculator, transport

    def Setup(self, flow: "FiniteVolumeSolver"):
        if self.fluxCalculator is not None:
            flow.RegisterRHSFunction("CompactCompressibleNSSpeciesTransport::AdvectionFlux", self.fluxCalculator)
        if self.transport is not None:
            flow.RegisterRHSFunction("CompactCompressibleNSSpeciesTransport::DiffusionFlux", self.transport)


# ---------------------------------------------------------------------------------------------
# solver
# ---------------------------------------------------------------------------------------------
LIMITERS = {"none": L.LIMITER_NONE, "zero": L.LIMITER_ZERO, "minmod": L.LIMITER_MINMOD, "vanleer": L.LIMITER_VANLEER,
            "vanalbada": L.LIMITER_VANALBADA, "sin": L.LIMITER_SIN}


def make_physics(eos, processes, petscfv_type: str = "upwind", limiter: str = "none", maxLimGrad: float = 1e10):
    """Build the abl_physics_desc the processes register. Returns (desc, keep-alive list)."""
    p = L.PhysicsDesc()
    keep: list = []
    eos._fill(p, keep)
    p.n_species = len(eos.GetSpeciesVariables())
    p.pgs_alpha = 1.0
    p.max_lim_grad = maxLimGrad
    p.reconstruction = L.RECON_LEASTSQUARES if petscfv_type == "leastsquares" else L.RECON_UPWIND
    p.limiter = LIMITERS[limiter]
    p.transport = L.TRANSPORT_NONE
    flux = None
    for proc in processes:
        if isinstance(proc, NavierStokesTransport):
            if proc.fluxCalculator is not None:
                p.advection = 1
                flux = proc.fluxCalculator
            if proc.transport is not None:
                p.diffusion = 1
                proc.transport._fill(p)
        elif isinstance(proc, SpeciesTransport):
            if not eos.GetSpeciesVariables():
                continue
            if proc.fluxCalculator is not None:
                p.species_advection = 1
                if flux is not None and type(flux) is not type(proc.fluxCalculator):
                    raise ValueError("NavierStokesTransport and SpeciesTransport must share one flux calculator type")
                flux = proc.fluxCalculator
            if proc.transport is not None:
                p.species_diffusion = 1
                proc.transport._fill(p)
        elif isinstance(proc, CompactCompressibleNSSpeciesTransport):
            species = bool(eos.GetSpeciesVariables())
            if proc.fluxCalculator is not None:
                if flux is not None and type(flux) is not type(proc.fluxCalculator):
                    raise ValueError("processes must share one flux calculator type")
                flux = proc.fluxCalculator
                p.advection = 1
                p.species_advection = int(species)
                p.species_advection_compact = int(species)
            if proc.transport is not None:
                p.diffusion = 1
                p.species_diffusion = int(species)
                proc.transport._fill(p)
    if flux is not None:
        p.flux = flux.kind
        minf, alpha, gamma = flux._params()
        p.ausmpup_minf = minf
        p.pgs_alpha = alpha
    return p, keep


class FiniteVolumeSolver:
    """Owns one abl_fv handle: mesh + geometry + weights resident on one GPU."""

    def __init__(self, mesh, eos, processes, petscfv_type: str = "upwind", limiter: str = "none", maxLimGrad: float = 1e10,
                 device: int = 0):
        self.mesh = mesh
        self.eos = eos
        self.processes = list(processes)
        self.registered: list[str] = []
        for proc in self.processes:
            proc.Setup(self)
        self.physics, self._keep = make_physics(eos, self.processes, petscfv_type, limiter, maxLimGrad)
        desc = mesh.desc()
        h = C.c_void_p()
        L.check(L.lib.abl_fv_create(C.byref(desc), C.byref(self.physics), device, C.byref(h)), "abl_fv_create")
        self.handle = h
        nc, na, ncell, nf = (C.c_int32() for _ in range(4))
        L.check(L.lib.abl_fv_sizes(h, C.byref(nc), C.byref(na), C.byref(ncell), C.byref(nf)))
        self.nc, self.naux, self.n_cells, self.n_faces = nc.value, na.value, ncell.value, nf.value
        self._n_bc = 1  # every ghost is outflow until SetBoundary
        self.device = device

    def RegisterRHSFunction(self, name: str, obj):
        self.registered.append(name)

    def ComputeRHSFunction(self, time: float, locX: np.ndarray, locF: np.ndarray, precision: int = L.PRECISION_FP64):
        """locF += RHS(locX) with host arrays (n_cells, nc)."""
        assert locX.shape == (self.n_cells, self.nc) and locF.shape == locX.shape
        x = np.ascontiguousarray(locX, dtype=np.float64)
        assert locF.dtype == np.float64 and locF.flags.c_contiguous
        L.check(L.lib.abl_fv_rhs_host(self.handle, time, L.dptr(x), L.dptr(locF), precision), "abl_fv_rhs_host")
        return locF

    def ComputeRHSDevice(self, time: float, U_ptr: int, F_ptr: int, precision: int = L.PRECISION_FP64, stream: int = 0):
        """F += RHS(U) with device pointers (e.g. torch tensors' data_ptr()), enqueued on `stream`."""
        L.check(L.lib.abl_fv_rhs(self.handle, time, C.c_void_p(U_ptr), C.c_void_p(F_ptr), precision, C.c_void_p(stream)), "abl_fv_rhs")

    def ComputeRHSPhaseDevice(self, time: float, U_ptr: int, F_ptr: int, phase: int, precision: int = L.PRECISION_FP64, stream: int = 0):
        """One phase of a split RHS (L.RHS_PHASE_INTERIOR reads no halo row; L.RHS_PHASE_REST, after the
        halo rows are current, finishes it): the two in order equal ComputeRHSDevice."""
        L.check(L.lib.abl_fv_rhs_phase(self.handle, time, C.c_void_p(U_ptr), C.c_void_p(F_ptr), precision, phase, C.c_void_p(stream)),
                "abl_fv_rhs_phase")

    def ComputeJVP(self, time: float, locX: np.ndarray, dX: np.ndarray, dF: np.ndarray, F: np.ndarray | None = None):
        """dF += J(locX) dX (and F += RHS(locX) when F is given), host arrays (n_cells, nc)."""
        x = np.ascontiguousarray(locX, dtype=np.float64)
        dx = np.ascontiguousarray(dX, dtype=np.float64)
        assert dF.dtype == np.float64 and dF.flags.c_contiguous
        L.check(L.lib.abl_fv_jvp_host(self.handle, time, L.dptr(x), L.dptr(dx), L.dptr(F) if F is not None else None, L.dptr(dF)),
                "abl_fv_jvp_host")
        return dF

    def ComputeJVPDevice(self, time: float, U_ptr: int, dU_ptr: int, dF_ptr: int, F_ptr: int = 0, stream: int = 0):
        L.check(L.lib.abl_fv_jvp(self.handle, time, C.c_void_p(U_ptr), C.c_void_p(dU_ptr), C.c_void_p(F_ptr or None), C.c_void_p(dF_ptr),
                                 C.c_void_p(stream)), "abl_fv_jvp")

    def SetJVPMode(self, mode: int):
        """L.JVP_EXACT (default) or L.JVP_FROZEN_LIMITER for the following JVP calls."""
        L.check(L.lib.abl_fv_set_jvp_mode(self.handle, int(mode)), "abl_fv_set_jvp_mode")

    def ComputeVJP(self, time: float, locX: np.ndarray, Fbar: np.ndarray, Ubar: np.ndarray):
        """Ubar += J(locX)^T Fbar, host arrays (n_cells, nc); Fbar is read on owned cells."""
        x = np.ascontiguousarray(locX, dtype=np.float64)
        fb = np.ascontiguousarray(Fbar, dtype=np.float64)
        assert Ubar.dtype == np.float64 and Ubar.flags.c_contiguous and Ubar.shape == x.shape
        L.check(L.lib.abl_fv_vjp_host(self.handle, time, L.dptr(x), L.dptr(fb), L.dptr(Ubar)), "abl_fv_vjp_host")
        return Ubar

    def ComputeVJPDevice(self, time: float, U_ptr: int, Fbar_ptr: int, Ubar_ptr: int, stream: int = 0):
        L.check(L.lib.abl_fv_vjp(self.handle, time, C.c_void_p(U_ptr), C.c_void_p(Fbar_ptr), C.c_void_p(Ubar_ptr), C.c_void_p(stream)),
                "abl_fv_vjp")

    # ---- the steps around the RHS (boundary ghosts, CFL step, explicit steps) ----------------------
    def SetBoundary(self, table, cell_bc=None):
        """Ghost-cell conditions: table = [(kind, value or None, enforce_at_face), ...] with kind one of
        L.BC_*; cell_bc[c] = the entry of boundary ghost c (None: entry 0 for every ghost)."""
        arr = (L.BoundaryCondition * len(table))()
        for i, (kind, value, enforce) in enumerate(table):
            arr[i].kind = int(kind)
            arr[i].enforce_at_face = int(bool(enforce))
            if value is not None:
                for k, v in enumerate(value):
                    arr[i].value[k] = float(v)
        cb = None if cell_bc is None else np.ascontiguousarray(cell_bc, dtype=np.int32)
        L.check(L.lib.abl_fv_set_boundary(self.handle, len(table), C.cast(arr, C.c_void_p), L.iptr(cb) if cb is not None else None),
                "abl_fv_set_boundary")
        self._n_bc = len(table)

    def FillGhostsDevice(self, U_ptr: int, stream: int = 0):
        L.check(L.lib.abl_fv_fill_ghosts(self.handle, 0.0, C.c_void_p(U_ptr), C.c_void_p(stream)), "abl_fv_fill_ghosts")

    def FillGhostsJVPDevice(self, dU_ptr: int, stream: int = 0):
        """Tangent of the ghost fill on a perturbation (in place)."""
        L.check(L.lib.abl_fv_fill_ghosts_jvp(self.handle, C.c_void_p(dU_ptr), C.c_void_p(stream)), "abl_fv_fill_ghosts_jvp")

    def FillGhostsVJPDevice(self, Ubar_ptr: int, stream: int = 0) -> np.ndarray:
        """Adjoint of the ghost fill on adjoint rows (in place); returns the adjoint of every condition's
        value, shape (number of conditions, L.BC_MAX_COMPONENTS)."""
        vb = np.zeros((self._n_bc, L.BC_MAX_COMPONENTS))
        L.check(L.lib.abl_fv_fill_ghosts_vjp(self.handle, C.c_void_p(Ubar_ptr), vb.ctypes.data_as(C.c_void_p), C.c_void_p(stream)),
                "abl_fv_fill_ghosts_vjp")
        return vb

    def SetPressureFunctional(self, cells, weights):
        """J(U) = sum_j weights[j] p(U[cells[j]]); repeated cells are merged (their weights added)."""
        cells = np.asarray(cells, dtype=np.int64)
        weights = np.asarray(weights, dtype=np.float64)
        uc, inv = np.unique(cells, return_inverse=True)
        w = np.zeros(uc.size)
        np.add.at(w, inv, weights)
        c32 = np.ascontiguousarray(uc, dtype=np.int32)
        L.check(L.lib.abl_fv_set_pressure_functional(self.handle, c32.size, L.iptr(c32), w.ctypes.data_as(C.c_void_p)),
                "abl_fv_set_pressure_functional")

    def PressureFunctionalDevice(self, U_ptr: int, Ubar_ptr: int = 0, stream: int = 0) -> float:
        """J at the device state; with Ubar_ptr, dJ/dU is added into those rows."""
        J = C.c_double(0.0)
        L.check(L.lib.abl_fv_pressure_functional(self.handle, C.c_void_p(U_ptr), C.byref(J), C.c_void_p(Ubar_ptr or None),
                                                 C.c_void_p(stream)), "abl_fv_pressure_functional")
        return J.value

    def CflTimeStepDevice(self, U_ptr: int, cfl: float, stream: int = 0) -> float:
        dt = C.c_double(0.0)
        L.check(L.lib.abl_fv_cfl_dt(self.handle, C.c_void_p(U_ptr), float(cfl), C.byref(dt), C.c_void_p(stream)), "abl_fv_cfl_dt")
        return dt.value

    def RkStageDevice(self, a: float, U0_ptr: int, b: float, Us_ptr: int, dt: float, F_ptr: int, Uout_ptr: int, stream: int = 0):
        """Uout = a U0 + b (Us + dt F) on the owned rows (a == 0 drops U0)."""
        L.check(L.lib.abl_fv_rk_stage(self.handle, float(a), C.c_void_p(U0_ptr or None), float(b), C.c_void_p(Us_ptr), float(dt),
                                      C.c_void_p(F_ptr), C.c_void_p(Uout_ptr), C.c_void_p(stream)), "abl_fv_rk_stage")

    def NormalizeSpeciesDevice(self, U_ptr: int, stream: int = 0):
        L.check(L.lib.abl_fv_normalize_species(self.handle, C.c_void_p(U_ptr), C.c_void_p(stream)), "abl_fv_normalize_species")

    def StepDevice(self, scheme: int, time: float, dt: float, U_ptr: int, precision: int = L.PRECISION_FP64, stream: int = 0):
        L.check(L.lib.abl_fv_step(self.handle, scheme, time, dt, C.c_void_p(U_ptr), precision, C.c_void_p(stream)), "abl_fv_step")

    def StepCflDevice(self, scheme: int, cfl: float, U_ptr: int, precision: int = L.PRECISION_FP64, time_ptr: int = 0, stream: int = 0):
        """One step with dt = the CFL step of the current state, computed and used on the device (no
        host synchronisation); dt is added to the device double at time_ptr when given."""
        L.check(L.lib.abl_fv_step_cfl(self.handle, scheme, float(cfl), C.c_void_p(U_ptr), precision, C.c_void_p(time_ptr or None),
                                      C.c_void_p(stream)), "abl_fv_step_cfl")

    def IntegrateDevice(self, U_ptr: int, t_end: float, cfl: float, scheme: int = L.STEP_EULER, precision: int = L.PRECISION_FP64,
                        dt0: float = 0.1, stream: int = 0) -> int:
        """March the device state to t_end as the reference's TimeStepper does with ts_adapt_type physics:
        first step min(dt0, CFL step); after each step the next one is the CFL step of the state that step
        started from (PETSc's adaptor runs before the solution takes the update), cut so the march ends
        exactly at t_end without a sliver of a last step (TS_EXACTFINALTIME_MATCHSTEP, src/solver/
        timeStepper.cpp:37; src/solver/adaptPhysics.cpp:3-24). Returns the number of steps."""
        def match(h, t):
            hmax = t_end - t
            if t < t_end and t + h > t_end:
                h = hmax
            if t < t_end and t + h < t_end and h * 2.0 > hmax:
                h = hmax / 2.0
            if t < t_end and t + h < t_end and h * 1.01 > hmax:
                h = hmax
            return h

        self.FillGhostsDevice(U_ptr, stream)
        t, n = 0.0, 0
        dt = match(min(dt0, self.CflTimeStepDevice(U_ptr, cfl, stream)), t)
        while t < t_end:
            nxt = self.CflTimeStepDevice(U_ptr, cfl, stream)
            self.StepDevice(scheme, t, dt, U_ptr, precision, stream)
            t = t_end if t + dt >= t_end or t_end - (t + dt) <= 1e-12 * t_end else t + dt
            n += 1
            dt = match(nxt, t)
        return n

    # ---- output and restart: the owned rows (the PETSc global vector of this rank) -----------------
    def DownloadOwnedDevice(self, src_ptr: int, width: int | None = None, stream: int = 0) -> np.ndarray:
        """Owned rows of a device array (state by default; width = naux for the aux fields), ascending
        local cell order."""
        width = self.nc if width is None else int(width)
        n = int(np.count_nonzero(np.asarray(self.mesh.cell_kind) == L.CELL_OWNED))
        out = np.empty((n, width))
        L.check(L.lib.abl_fv_download_owned(self.handle, C.c_void_p(src_ptr), width, out.ctypes.data_as(C.c_void_p), C.c_void_p(stream)),
                "abl_fv_download_owned")
        return out

    def UploadOwnedDevice(self, rows: np.ndarray, dst_ptr: int, stream: int = 0):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        L.check(L.lib.abl_fv_upload_owned(self.handle, rows.ctypes.data_as(C.c_void_p), rows.shape[1], C.c_void_p(dst_ptr), C.c_void_p(stream)),
                "abl_fv_upload_owned")

    def UpdateAux(self, locX: np.ndarray):
        """Recompute the aux fields (T, u, Y) from host state locX (CellSolver::UpdateAuxFields)."""
        x = np.ascontiguousarray(locX, dtype=np.float64)
        L.check(L.lib.abl_fv_update_aux_host(self.handle, L.dptr(x)), "abl_fv_update_aux_host")

    def GetAux(self) -> np.ndarray:
        a = np.zeros((self.n_cells, self.naux))
        L.check(L.lib.abl_fv_get_aux(self.handle, L.dptr(a)))
        return a

    def SetAux(self, aux: np.ndarray):
        a = np.ascontiguousarray(aux, dtype=np.float64)
        L.check(L.lib.abl_fv_set_aux(self.handle, L.dptr(a)))

    def Status(self) -> int:
        return L.lib.abl_fv_status(self.handle)

    def Profile(self, enable: bool = True):
        L.check(L.lib.abl_fv_profile(self.handle, int(enable)))

    def ProfileRead(self) -> dict:
        """Per-kernel device milliseconds of the last ComputeRHS* call (profiling must be on)."""
        n = C.c_int32()
        ms = (C.c_float * 8)()
        names = C.create_string_buffer(32 * 8)
        L.check(L.lib.abl_fv_profile_read(self.handle, C.byref(n), ms, names))
        raw = names.raw
        return {raw[32 * i:32 * (i + 1)].split(b"\0")[0].decode(): float(ms[i]) for i in range(n.value)}

    def LaunchCount(self, precision: int = L.PRECISION_FP64) -> int:
        n = C.c_int32()
        L.check(L.lib.abl_fv_launch_count(self.handle, precision, C.byref(n)))
        return n.value

    def RecordClasses(self) -> tuple[int, int]:
        """(weight classes, geometry classes) of the device layout: the distinct per-cell cone weight
        sequences and tile face geometry records stored once, 0 where every cell / face has its own."""
        w, g = C.c_int32(), C.c_int32()
        L.check(L.lib.abl_fv_record_classes(self.handle, C.byref(w), C.byref(g)))
        return w.value, g.value

    def FusedInfo(self) -> dict:
        """Which RHS kernels the handle runs: the fused one-pass kernel per precision (where a tile fits
        in shared memory), its distinct tile tables, and the most cells one tile stages."""
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        L.check(L.lib.abl_fv_fused_info(self.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return {"fp64": bool(a.value), "mixed": bool(b.value), "tile_classes": c.value, "max_staged_cells": d.value}

    def close(self):
        if getattr(self, "handle", None):
            L.lib.abl_fv_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def eos_property(physics: L.PhysicsDesc, dim: int, prop: int, conserved: np.ndarray, T: np.ndarray | None = None) -> np.ndarray:
    """Device batch of a ThermodynamicFunction (T is None) or ThermodynamicTemperatureFunction."""
    conserved = np.ascontiguousarray(conserved, dtype=np.float64)
    n = conserved.shape[0]
    ps = physics.n_species if prop == L.PROP_SPECIES_SENSIBLE_ENTHALPY else 1
    out = np.zeros((n, max(ps, 1)))
    Ta = None if T is None else np.ascontiguousarray(T, dtype=np.float64)
    L.check(L.lib.abl_eos_batch(C.byref(physics), dim, prop, n, L.dptr(conserved), L.dptr(Ta), L.dptr(out)), "abl_eos_batch")
    return out
