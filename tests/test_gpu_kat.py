"""The device physics (flux calculators, EOS) against the reference's known-answer vectors and the
oracle, through the C ABI batch entry points."""
import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from oracle import oracle as orc
from tests import golden_cases as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [c for c, _, _ in G.flux_cases()], ids=lambda c: c["name"])
def test_device_flux_calculator_kat(case):
    kind = G.FLUX_KINDS[case["kind"]]
    n = len(case["uL"])
    args = [np.array(case[k][:n]) for k in ("uL", "aL", "rhoL", "pL", "uR", "aR", "rhoR", "pR")]
    calc = {"ausm": fv.Ausm(), "average": fv.AverageFlux(), "off": fv.OffFlux(),
            "riemann": fv.Riemann(fv.PerfectGas({"gamma": case.get("gamma", 1.4)})),
            "ausmpup": fv.AusmpUp(case.get("minf", 0.0), fv.PressureGradientScaling(None, case.get("pgs_alpha", 1.0)))}[case["kind"]]
    mf, p12, d = calc.GetFluxCalculatorFunction()(*args)
    np.testing.assert_array_equal(d, case["expectedDirection"][:n])
    np.testing.assert_allclose(mf, case["expectedMassFlux"][:n], rtol=0, atol=1e-2)
    np.testing.assert_allclose(p12, case["expectedInterfacePressure"][:n], rtol=0, atol=1.0)
    # and bit-for-bit-level agreement with the oracle
    omf, op12, od = orc.flux_calculator(kind, *args, minf=case.get("minf", 0.0), pgs_alpha=case.get("pgs_alpha", 1.0),
                                        gamma=case.get("gamma", 1.4))
    np.testing.assert_array_equal(d, od)
    np.testing.assert_allclose(mf, omf, rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(p12, op12, rtol=1e-13, atol=1e-9)


@pytest.mark.parametrize("kind", [L.FLUX_AUSM, L.FLUX_AUSMPUP, L.FLUX_RIEMANN, L.FLUX_AVERAGE])
def test_device_flux_calculator_random(kind):
    rng = np.random.default_rng(kind)
    n = 4096
    rhoL, rhoR = rng.uniform(0.1, 5, n), rng.uniform(0.1, 5, n)
    pL, pR = rng.uniform(1e3, 4e5, n), rng.uniform(1e3, 4e5, n)
    aL, aR = np.sqrt(1.4 * pL / rhoL), np.sqrt(1.4 * pR / rhoR)
    uL, uR = rng.uniform(-600, 600, n), rng.uniform(-600, 600, n)
    args = (uL, aL, rhoL, pL, uR, aR, rhoR, pR)
    mf = np.zeros(n); p12 = np.zeros(n); d = np.zeros(n, np.int32)
    L.check(L.lib.abl_flux_calculator_batch(kind, 0.3, 1.0, 1.4, n, *[L.dptr(np.ascontiguousarray(a)) for a in args], L.dptr(mf),
                                            L.dptr(p12), L.iptr(d)))
    omf, op12, od = orc.flux_calculator(kind, *args, minf=0.3, pgs_alpha=1.0, gamma=1.4)
    np.testing.assert_array_equal(d, od)
    np.testing.assert_allclose(mf, omf, rtol=1e-11, atol=1e-9)
    np.testing.assert_allclose(p12, op12, rtol=1e-11, atol=1e-6)


@pytest.mark.parametrize("idx", range(len(G.load("perfect_gas.json")["cases"])))
def test_device_perfect_gas_kat(idx):
    c, phys, dim, prop, u = list(G.perfect_gas_cases())[idx]
    direct = fv.eos_property(phys, dim, prop, u)[0]
    np.testing.assert_allclose(direct[:len(c["expectedValue"])], c["expectedValue"], rtol=0, atol=1e-6)
    T = fv.eos_property(phys, dim, L.PROP_TEMPERATURE, u)[0, 0]
    if c["expectedTemperature"] is not None:
        assert abs(T - c["expectedTemperature"]) < 1e-6
    withT = fv.eos_property(phys, dim, prop, u, T=np.array([T]))[0]
    np.testing.assert_allclose(withT[:len(c["expectedValue"])], c["expectedValue"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("idx", range(len(G.load("tchem_gri30.json")["cases"])))
def test_device_tchem_gri30_kat(idx):
    c, phys, keep, dim, u = list(G.tchem_cases())[idx]
    T = fv.eos_property(phys, dim, L.PROP_TEMPERATURE, u)[0, 0]
    Tor = orc.eos(phys, dim, L.PROP_TEMPERATURE, u)[0, 0]
    assert abs(T - Tor) <= 1e-9 * Tor
    if c["expectedTemperature"] is not None:
        assert abs(T - c["expectedTemperature"]) / c["expectedTemperature"] < 1e-5
    tol = c["errorTolerance"]
    for name, expected in c["testProperties"].items():
        prop = G.PROPS[name]
        for got in (fv.eos_property(phys, dim, prop, u)[0], fv.eos_property(phys, dim, prop, u, T=np.array([T]))[0]):
            for e, v in zip(expected, got):
                if e == 0:
                    assert abs(v) < tol * 1e6, (name, v)
                else:
                    assert abs((e - v) / (e + 1e-30)) < tol, (name, e, v)
