"""abl_eos_batch_noalloc: the allocation-free EOS batch for states already in device memory.

Its callers cannot allocate device memory during the call -- their HBM is reserved by a pool
allocator, or they evaluate properties inside a time step where the device-wide synchronisation of a
cudaFree is not affordable -- so the entry point keeps its species tables and status word in a small
static device array instead of per-call buffers. This file checks it through the C ABI against the
allocating entry point, abl_eos_batch, on two calls in a row (the second reuses the array the first
left behind). It is named to be collected last, and it creates its own device buffers, so it runs the
same alone in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from ablate_b200 import _lib as L
from ablate_b200 import fv
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, the FP64 parity tolerance of the other device tests


def _noalloc(torch, physics, dim, prop, U, T=None):
    dev = torch.device("cuda", 0)
    n = U.shape[0]
    size = physics.n_species if prop == L.PROP_SPECIES_SENSIBLE_ENTHALPY else 1
    u = torch.from_numpy(np.ascontiguousarray(U)).to(dev)
    t = None if T is None else torch.from_numpy(np.ascontiguousarray(T, dtype=np.float64)).to(dev)
    out = torch.full((n, max(size, 1)), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = L.lib.abl_eos_batch_noalloc(C.byref(physics), dim, prop, n, C.c_void_p(u.data_ptr()),
                                     C.c_void_p(t.data_ptr()) if t is not None else None, C.c_void_p(out.data_ptr()),
                                     C.c_void_p(stream.cuda_stream))
    L.check(rc, "abl_eos_batch_noalloc")
    return out.cpu().numpy()


def _close(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    assert np.all(np.abs(a - b) <= TOL * scale + 1e-300), np.max(np.abs(a - b) / scale)


def test_noalloc_matches_allocating_batch_twice():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    # a NASA-7 mixture (the reference's gri30 known-answer states) and a perfect gas, each called twice
    cases = list(G.tchem_cases())
    rng = np.random.default_rng(7)
    for repeat in range(2):
        for c, phys, keep, dim, u in cases:
            U = np.repeat(u, 33, axis=0) * (1.0 + 1e-3 * rng.standard_normal((33, u.shape[1])))
            U = np.ascontiguousarray(U)
            for prop in (L.PROP_TEMPERATURE, L.PROP_PRESSURE, L.PROP_SPEED_OF_SOUND, L.PROP_SPECIES_SENSIBLE_ENTHALPY):
                ref = fv.eos_property(phys, dim, prop, U)
                got = _noalloc(torch, phys, dim, prop, U)
                _close(got, ref)
            T = fv.eos_property(phys, dim, L.PROP_TEMPERATURE, U)[:, 0]
            ref = fv.eos_property(phys, dim, L.PROP_INTERNAL_SENSIBLE_ENERGY, U, T)
            _close(_noalloc(torch, phys, dim, L.PROP_INTERNAL_SENSIBLE_ENERGY, U, T), ref)
        pg = G.perfect_gas_physics(1.4, 287.0)
        U = np.stack([rng.uniform(0.5, 2, 500), rng.uniform(2e5, 4e5, 500), rng.uniform(-50, 50, 500),
                      rng.uniform(-50, 50, 500), rng.uniform(-50, 50, 500)], 1)
        for prop in (L.PROP_PRESSURE, L.PROP_TEMPERATURE, L.PROP_SPEED_OF_SOUND):
            _close(_noalloc(torch, pg, 3, prop, U), fv.eos_property(pg, 3, prop, U))


def test_noalloc_rejects_more_species_than_its_scratch_holds():
    # 65 species pass the descriptor check (up to 128) and reach the entry point's own limit
    pg = G.perfect_gas_physics(1.4, 287.0, ns=65)
    rc = L.lib.abl_eos_batch_noalloc(C.byref(pg), 3, L.PROP_PRESSURE, 1, C.c_void_p(1), None, C.c_void_p(1), None)
    assert rc == L.ERR_INVALID_ARGUMENT
    assert b"its static scratch holds" in L.lib.abl_last_error_string()


def test_noalloc_zero_length_call_is_a_warm_up():
    # n = 0 resolves the scratch address (and so loads the device code) without launching anything
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    pg = G.perfect_gas_physics(1.4, 287.0)
    rc = L.lib.abl_eos_batch_noalloc(C.byref(pg), 3, L.PROP_PRESSURE, 0, None, None, None, None)
    L.check(rc, "abl_eos_batch_noalloc warm-up")
