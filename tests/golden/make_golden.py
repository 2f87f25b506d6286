"""Extract the reference's own known-answer vectors for the FV RHS path into JSON fixtures.

Reads the ABLATE unit-test sources as text (it does not build or run them) and writes
``tests/golden/*.json``. Run it where the reference checkout is available:

    python tests/golden/make_golden.py <reference checkout>

Sources read (ABLATE 0.13.03):
  tests/unitTests/finiteVolume/fluxCalculator/fluxCalculatorTests.cpp:56-403
  tests/unitTests/finiteVolume/processes/navierStokesTransportTests.cpp:56-121
  tests/unitTests/eos/perfectGasTests.cpp:91-236
  tests/unitTests/eos/tChemTests.cpp:259+           (+ tests/unitTests/inputs/eos/gri30.yaml NASA-7 data)
  tests/unitTests/eos/transport/sutherlandTests.cpp:143-145
  tests/unitTests/finiteVolume/compressibleShockTubeTests.cpp:210+
"""
from __future__ import annotations

import json
import math
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def _num(tok: str) -> float:
    tok = tok.strip()
    if not tok:
        raise ValueError("empty")
    if tok in ("NAN", "NaN"):
        return float("nan")
    # arithmetic such as "1.2 * 1E5", ".9 * -20", "1004.5 / 1.4"
    safe = re.sub(r"[^0-9eE+\-*/. ()]", "", tok)
    if safe != tok.replace(" ", "").replace("\t", "") and safe.replace(" ", "") != tok.replace(" ", ""):
        raise ValueError(f"unexpected token {tok!r}")
    return float(eval(safe, {"__builtins__": {}}, {}))


def _braced(text: str, start: int) -> tuple[str, int]:
    """Return the contents of the brace group opening at text[start] == '{' and the index after it."""
    assert text[start] == "{"
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start + 1:i], i + 1
    raise ValueError("unbalanced braces")


def _field(block: str, name: str) -> str | None:
    m = re.search(r"\." + name + r"\s*=\s*", block)
    if not m:
        return None
    i = m.end()
    # skip type prefixes like std::vector<PetscReal>
    m2 = re.match(r"std::vector<[^>]+>\s*", block[i:])
    if m2:
        i += m2.end()
    if block[i] == "{":
        inner, _ = _braced(block, i)
        return "{" + inner + "}"
    # expressions with parentheses (std::make_shared<...>(...)) may span lines: take the balanced group
    depth = 0
    for j in range(i, len(block)):
        ch = block[j]
        if ch in "(<{":
            depth += 1
        elif ch in ")>}":
            depth -= 1
        elif ch == "," and depth == 0:
            return block[i:j].strip()
        elif ch == "\n" and depth == 0:
            return block[i:j].strip()
    return block[i:].strip()


def _list(s: str) -> list[float]:
    s = s.strip()
    assert s.startswith("{") and s.endswith("}"), s
    inner = s[1:-1]
    return [_num(t) for t in inner.split(",") if t.strip()]


def _blocks(text: str, struct: str) -> list[str]:
    out = []
    for m in re.finditer(r"\(" + struct + r"\)\s*\{", text):
        inner, _ = _braced(text, m.end() - 1)
        out.append(inner)
    return out


DIRS = {"LEFT": 1, "RIGHT": 2, "NA": 0}


def flux_calculators(ref: Path) -> dict:
    src = (ref / "tests/unitTests/finiteVolume/fluxCalculator/fluxCalculatorTests.cpp").read_text()
    cases = []
    for b in _blocks(src, "FluxCalculatorTestParameters"):
        name = _field(b, "testName").strip('"')
        calc = _field(b, "fluxCalculator")
        entry = {"name": name, "source": "tests/unitTests/finiteVolume/fluxCalculator/fluxCalculatorTests.cpp"}
        if "Riemann2Gas" in calc or "RiemannStiff" in calc:
            continue  # two-gas / stiffened gas calculators are outside this backend's scope
        if "fluxCalculator::Ausm>" in calc:
            entry.update(kind="ausm")
        elif "AusmpUp" in calc:
            entry.update(kind="ausmpup", minf=0.0, pgs_alpha=100.0 if "PressureGradientScaling" in calc else 1.0)
        elif "AverageFlux" in calc:
            entry.update(kind="average")
        elif "OffFlux" in calc:
            entry.update(kind="off")
        elif "Riemann" in calc:
            g = re.search(r'"gamma",\s*"([0-9.]+)"', calc)
            entry.update(kind="riemann", gamma=float(g.group(1)) if g else 1.4)
        else:
            raise ValueError(calc)
        # the block text after the calculator: parse the vectors
        for key in ("uL", "aL", "rhoL", "pL", "uR", "aR", "rhoR", "pR", "expectedMassFlux", "expectedInterfacePressure"):
            entry[key] = _list(_field(b, key))
        dirs = _field(b, "expectedDirection")
        entry["expectedDirection"] = [DIRS[t.strip()] for t in dirs.strip("{}").split(",") if t.strip()]
        cases.append(entry)
    return {"tolerance": {"massFlux": 1e-2, "p12": 1.0}, "cases": cases}


def ns_transport(ref: Path) -> dict:
    src = (ref / "tests/unitTests/finiteVolume/processes/navierStokesTransportTests.cpp").read_text()
    adv = []
    for b in _blocks(src, "NavierStokesTransportFluxTestParameters"):
        assert "Ausm" in _field(b, "fluxCalculator")
        adv.append({"area": _list(_field(b, "area")), "xLeft": _list(_field(b, "xLeft")), "xRight": _list(_field(b, "xRight")),
                    "expectedFlux": _list(_field(b, "expectedFlux"))})
    stress = []
    for b in _blocks(src, "StressTensorTestParameters"):
        stress.append({"dim": int(_num(_field(b, "dim"))), "mu": _num(_field(b, "mu")), "gradVel": _list(_field(b, "gradVel")),
                       "expectedStressTensor": _list(_field(b, "expectedStressTensor"))})
    return {"source": "tests/unitTests/finiteVolume/processes/navierStokesTransportTests.cpp",
            "advection": {"fluxCalculator": "ausm", "eos": {"gamma": 1.4, "Rgas": 287.0}, "tolerance": 1e-3, "TempGuess": 300.0, "cases": adv},
            "stressTensor": {"tolerance": 1e-8, "cases": stress}}


PROPS = ["Pressure", "Temperature", "InternalSensibleEnergy", "SensibleEnthalpy", "SpecificHeatConstantVolume",
         "SpecificHeatConstantPressure", "SpeedOfSound", "SpeciesSensibleEnthalpy", "Density"]


def _fields(s: str) -> list[dict]:
    out = []
    for m in re.finditer(r'MockField::Create\("(\w+)",\s*(\d+)(?:,\s*(\d+))?\)', s):
        out.append({"name": m.group(1), "components": int(m.group(2)), "offset": int(m.group(3) or 0)})
    return out


def perfect_gas(ref: Path) -> dict:
    src = (ref / "tests/unitTests/eos/perfectGasTests.cpp").read_text()
    cases = []
    for b in _blocks(src, "PGTestParameters"):
        opts = dict(re.findall(r'\{"(\w+)",\s*"([0-9.eE+-]+)"\}', _field(b, "options")))
        prop = _field(b, "thermodynamicProperty").split("::")[-1]
        species = re.findall(r'"(\w+)"', _field(b, "species") or "")
        et = _field(b, "expectedTemperature")
        cases.append({"gamma": float(opts.get("gamma", 1.4)), "Rgas": float(opts.get("Rgas", 287.0)), "species": species,
                      "property": prop, "fields": _fields(_field(b, "fields")), "conservedValues": _list(_field(b, "conservedValues")),
                      "expectedTemperature": None if et in ("{}", None) else _num(et), "expectedValue": _list(_field(b, "expectedValue"))})
    return {"source": "tests/unitTests/eos/perfectGasTests.cpp", "tolerance": 1e-6, "cases": cases}


def sutherland(ref: Path) -> dict:
    src = (ref / "tests/unitTests/eos/transport/sutherlandTests.cpp").read_text()
    cases = []
    for b in _blocks(src, "SutherlandTransportTestParameters"):
        cases.append({k: _num(_field(b, k)) for k in ("temperatureIn", "densityIn", "cpIn", "expectedConductivity", "expectedViscosity",
                                                      "expectedDiffusivity")})
    return {"source": "tests/unitTests/eos/transport/sutherlandTests.cpp", "relativeTolerance": 1e-5, "cases": cases}


# --- NASA-7 data of the gri30 mechanism ----------------------------------------------------------
def _yaml_load(text: str):
    """YAML without the 1.1 implicit booleans (species 'NO' and element 'N' must stay strings)."""
    import yaml

    class Loader(yaml.SafeLoader):
        pass

    Loader.yaml_implicit_resolvers = {k: [(tag, rx) for tag, rx in v if tag != "tag:yaml.org,2002:bool"]
                                      for k, v in yaml.SafeLoader.yaml_implicit_resolvers.items()}
    return yaml.load(text, Loader=Loader)


def gri30_thermo(ref: Path) -> dict:
    doc = _yaml_load((ref / "tests/unitTests/inputs/eos/gri30.yaml").read_text())
    species = []
    for sp in doc["species"]:
        th = sp["thermo"]
        assert th["model"] == "NASA7"
        tr = th["temperature-ranges"]
        lo, hi = th["data"]
        assert len(tr) == 3
        species.append({"name": sp["name"], "composition": sp["composition"], "T_ranges": tr, "low": lo, "high": hi})
    phase_species = doc["phases"][0]["species"]
    order = [s["name"] for s in species]
    assert phase_species == order, "phase species order differs from the species list"
    return {"source": "tests/unitTests/inputs/eos/gri30.yaml", "species": species}


def tchem(ref: Path) -> dict:
    src = (ref / "tests/unitTests/eos/tChemTests.cpp").read_text()
    start = src.index("INSTANTIATE_TEST_SUITE_P(\n    TChemTests, TCThermodynamicPropertyTestFixture")
    end = src.index("INSTANTIATE_TEST_SUITE_P", start + 10)
    region = src[start:end]
    cases = []
    for b in _blocks(region, "TCTestParameters"):
        if "gri30.yaml" not in _field(b, "mechFile"):
            continue
        yimap = {k: _num(v) for k, v in re.findall(r'\{"([\w()]+)",\s*([0-9.eE+-]+)\}', _field(b, "yiMap"))}
        tp = _field(b, "testProperties")
        props = {}
        for m in re.finditer(r"ThermodynamicProperty::(\w+),\s*\{([^}]*)\}", tp):
            props[m.group(1)] = [_num(t) for t in m.group(2).split(",") if t.strip()]
        et = _field(b, "expectedTemperature")
        tol = _field(b, "errorTolerance")
        cases.append({"fields": _fields(_field(b, "fields")), "conservedEulerValues": _list(_field(b, "conservedEulerValues")),
                      "yiMap": yimap, "expectedTemperature": None if et in ("{}", None) else _num(et), "testProperties": props,
                      "errorTolerance": _num(tol) if tol else 1e-5})
    return {"source": "tests/unitTests/eos/tChemTests.cpp", "mechanism": "gri30", "cases": cases}


def shock_tube(ref: Path) -> dict:
    """1D shock tubes: initial states, AUSM, nx cells, CFL, final time, and the expected primitives."""
    src = (ref / "tests/unitTests/finiteVolume/compressibleShockTubeTests.cpp").read_text()
    cases = []
    for blk in _blocks(src, "CompressibleShockTubeParameters"):
        name = re.search(r'MpiTestParameter\("([^"]+)"', blk).group(1)
        ic_txt = _field(blk, "initialConditions")
        ic = {k: _num(v) for k, v in re.findall(r"\.(\w+)\s*=\s*([^,}]+)", ic_txt)}
        flux = re.search(r"fluxCalculator::(\w+)", _field(blk, "fluxCalculator")).group(1)
        ev_txt = _field(blk, "expectedValues")
        expected = {m.group(1): _list("{" + m.group(2) + "}") for m in re.finditer(r'\{"(\w+)",\s*\{([^}]*)\}\}', ev_txt)}
        cases.append({"name": name, "initial": ic, "flux": flux, "nx": int(_num(_field(blk, "nx"))), "maxTime": _num(_field(blk, "maxTime")),
                      "cfl": _num(_field(blk, "cfl")), "expected": expected})
    return {"source": "tests/unitTests/finiteVolume/compressibleShockTubeTests.cpp",
            "harness": "1D box [0, length], ghost cells holding the initial left/right state by face position, TS with "
                       "ts_adapt_type physics, ts_adapt_safety 1, ts_exact_final_time matchstep, ASSERT_NEAR 1e-6",
            "cases": cases}


def main(argv):
    if len(argv) < 2:
        print("usage: python tests/golden/make_golden.py <reference checkout>", file=sys.stderr)
        return 2
    ref = Path(argv[1])
    out = {
        "flux_calculators.json": flux_calculators(ref),
        "ns_transport.json": ns_transport(ref),
        "perfect_gas.json": perfect_gas(ref),
        "sutherland.json": sutherland(ref),
        "tchem_gri30.json": tchem(ref),
        "gri30_nasa7.json": gri30_thermo(ref),
        "shock_tube.json": shock_tube(ref),
    }
    for name, data in out.items():
        text = json.dumps(data, indent=1, allow_nan=True)
        (HERE / name).write_text(text + "\n")
        print(f"wrote {name}: {len(text)} bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
