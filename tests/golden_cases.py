"""Shared loaders that turn the golden JSON fixtures into call arguments (used by CPU and GPU tests)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from ablate_b200 import _lib as L
from ablate_b200 import fv

GOLDEN = Path(__file__).resolve().parent / "golden"

FLUX_KINDS = {"ausm": L.FLUX_AUSM, "ausmpup": L.FLUX_AUSMPUP, "average": L.FLUX_AVERAGE, "off": L.FLUX_OFF, "riemann": L.FLUX_RIEMANN}
PROPS = {"Pressure": L.PROP_PRESSURE, "Temperature": L.PROP_TEMPERATURE, "InternalSensibleEnergy": L.PROP_INTERNAL_SENSIBLE_ENERGY,
         "SensibleEnthalpy": L.PROP_SENSIBLE_ENTHALPY, "SpecificHeatConstantVolume": L.PROP_CV,
         "SpecificHeatConstantPressure": L.PROP_CP, "SpeedOfSound": L.PROP_SPEED_OF_SOUND,
         "SpeciesSensibleEnthalpy": L.PROP_SPECIES_SENSIBLE_ENTHALPY, "Density": L.PROP_DENSITY}


def load(name):
    return json.loads((GOLDEN / name).read_text())


def flux_cases():
    for c in load("flux_calculators.json")["cases"]:
        n = len(c["uL"])
        args = [np.array(c[k][:n], dtype=np.float64) for k in ("uL", "aL", "rhoL", "pL", "uR", "aR", "rhoR", "pR")]
        yield c, FLUX_KINDS[c["kind"]], args


def perfect_gas_physics(gamma, rgas, ns=0):
    p = L.PhysicsDesc()
    p.eos = L.EOS_PERFECT_GAS
    p.gamma = gamma
    p.r_gas = rgas
    p.n_species = ns
    return p


def perfect_gas_cases():
    for c in load("perfect_gas.json")["cases"]:
        euler = [f for f in c["fields"] if f["name"] == "euler"][0]
        vals = np.array(c["conservedValues"], dtype=np.float64)
        conserved = vals[euler["offset"]:euler["offset"] + euler["components"]]
        dim = euler["components"] - 2
        phys = perfect_gas_physics(c["gamma"], c["Rgas"], len(c["species"]))
        # species slots (zero) appended after euler so the state has the full layout
        u = np.concatenate([conserved, np.zeros(len(c["species"]))])[None, :]
        yield c, phys, dim, PROPS[c["property"]], u


def gri30_eos():
    thermo = load("gri30_nasa7.json")["species"]
    return fv.TChem(thermo)


def tchem_cases(eos=None):
    eos = eos or gri30_eos()
    names = eos.GetSpeciesVariables()
    phys, keep = fv.make_physics(eos, [])
    for c in load("tchem_gri30.json")["cases"]:
        euler = [f for f in c["fields"] if f["name"] == "euler"][0]
        dim = euler["components"] - 2
        ev = np.array(c["conservedEulerValues"][:euler["components"]], dtype=np.float64)
        rho = ev[0]
        y = np.zeros(len(names))
        for sp, val in c["yiMap"].items():
            y[names.index(sp)] = val
        u = np.concatenate([ev, rho * y])[None, :]
        yield c, phys, keep, dim, u
