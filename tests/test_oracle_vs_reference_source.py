"""The oracle's flux calculators against the reference's own source files (AUSM, AUSM+up, average,
off, exact Riemann core), compiled unchanged by `make -C oracle ref` into oracle/_ref. Skipped where
that library was not built (it needs the reference checkout at build time)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from ablate_b200 import _lib as L
from oracle import oracle as orc

REF_LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libablate_ref_flux.so"

pytestmark = pytest.mark.skipif(not REF_LIB.exists(), reason="oracle/_ref not built (needs the reference sources)")


def _ref():
    lib = C.CDLL(str(REF_LIB))
    dp = C.POINTER(C.c_double)
    lib.ref_flux_calculator_batch.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_long] + [dp] * 10 + [C.POINTER(C.c_int)]
    return lib, dp


@pytest.mark.parametrize("kind", [L.FLUX_OFF, L.FLUX_AVERAGE, L.FLUX_AUSM, L.FLUX_AUSMPUP, L.FLUX_RIEMANN])
@pytest.mark.parametrize("alpha", [1.0, 7.0])
def test_oracle_flux_matches_reference_source(kind, alpha):
    lib, dp = _ref()
    rng = np.random.default_rng(100 + kind)
    n = 20000
    rhoL, rhoR = rng.uniform(0.1, 5, n), rng.uniform(0.1, 5, n)
    pL, pR = rng.uniform(1e3, 4e5, n), rng.uniform(1e3, 4e5, n)
    aL, aR = np.sqrt(1.4 * pL / rhoL), np.sqrt(1.4 * pR / rhoR)
    uL, uR = rng.uniform(-600, 600, n), rng.uniform(-600, 600, n)
    args = [np.ascontiguousarray(a) for a in (uL, aL, rhoL, pL, uR, aR, rhoR, pR)]
    mf, p12, d = np.zeros(n), np.zeros(n), np.zeros(n, np.int32)
    rc = lib.ref_flux_calculator_batch(kind, 0.3, alpha, 1.4, n, *[a.ctypes.data_as(dp) for a in args], mf.ctypes.data_as(dp),
                                       p12.ctypes.data_as(dp), d.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 0
    omf, op12, od = orc.flux_calculator(kind, *args, minf=0.3, pgs_alpha=alpha, gamma=1.4)
    np.testing.assert_array_equal(od, d)
    np.testing.assert_allclose(omf, mf, rtol=1e-13, atol=1e-11)
    np.testing.assert_allclose(op12, p12, rtol=1e-13, atol=1e-8)
