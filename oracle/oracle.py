"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/liborc.so).

Imported only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, as the checker or
the timed CPU baseline; never by the product package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ablate_b200 import _lib as L

LIB_PATH = Path(__file__).resolve().parent / "liborc.so"


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ablate_b200/build.py`")
    lib = C.CDLL(str(LIB_PATH))
    dp, ip = L._dp, L._ip
    lib.orc_flux_calculator_batch.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int64] + [dp] * 10 + [ip]
    lib.orc_flux_calculator_batch.restype = C.c_int
    lib.orc_eos_batch.argtypes = [C.POINTER(L.PhysicsDesc), C.c_int, C.c_int, C.c_int64, dp, dp, dp]
    lib.orc_eos_batch.restype = C.c_int
    lib.orc_stress_tensor.argtypes = [C.c_int, C.c_double, dp, dp]
    lib.orc_stress_tensor.restype = C.c_int
    lib.orc_ns_advection_flux.argtypes = [C.POINTER(L.PhysicsDesc), C.c_int, dp, dp, dp, C.c_double, C.c_double, dp]
    lib.orc_ns_advection_flux.restype = C.c_int
    lib.orc_species_advection_flux.argtypes = [C.POINTER(L.PhysicsDesc), C.c_int, dp, dp, dp, C.c_double, C.c_double, dp]
    lib.orc_species_advection_flux.restype = C.c_int
    lib.orc_limiter.argtypes = [C.c_int, C.c_double]
    lib.orc_limiter.restype = C.c_double
    lib.orc_lsq_face_weights.argtypes = [C.POINTER(L.MeshDesc), dp]
    lib.orc_lsq_face_weights.restype = C.c_int
    lib.orc_rhs.argtypes = [C.POINTER(L.MeshDesc), C.POINTER(L.PhysicsDesc), dp, dp, dp, C.c_int]
    lib.orc_rhs.restype = C.c_int
    lib.orc_create.argtypes = [C.POINTER(L.MeshDesc), C.POINTER(L.PhysicsDesc)]
    lib.orc_create.restype = C.c_void_p
    lib.orc_run.argtypes = [C.c_void_p, dp, dp, dp, C.c_int]
    lib.orc_run.restype = C.c_int
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_destroy.restype = None
    lib.orc_last_error.restype = C.c_char_p
    return lib


lib = _load()


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed [{rc}]: {lib.orc_last_error().decode()}")


def flux_calculator(kind, uL, aL, rhoL, pL, uR, aR, rhoR, pR, minf=0.0, pgs_alpha=1.0, gamma=1.4):
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (uL, aL, rhoL, pL, uR, aR, rhoR, pR)]
    n = arrs[0].size
    mf = np.zeros(n)
    p12 = np.zeros(n)
    d = np.zeros(n, np.int32)
    _check(lib.orc_flux_calculator_batch(kind, minf, pgs_alpha, gamma, n, *[L.dptr(a) for a in arrs],
                                         L.dptr(mf), L.dptr(p12), L.iptr(d)), "flux calculator")
    return mf, p12, d


def eos(physics: L.PhysicsDesc, dim: int, prop: int, conserved: np.ndarray, T=None):
    conserved = np.ascontiguousarray(conserved, dtype=np.float64)
    n = conserved.shape[0]
    ps = physics.n_species if prop == L.PROP_SPECIES_SENSIBLE_ENTHALPY else 1
    out = np.zeros((n, max(ps, 1)))
    Ta = None if T is None else np.ascontiguousarray(T, dtype=np.float64)
    _check(lib.orc_eos_batch(C.byref(physics), dim, prop, n, L.dptr(conserved), L.dptr(Ta), L.dptr(out)), "eos")
    return out


def stress_tensor(dim, mu, grad_vel):
    g = np.ascontiguousarray(grad_vel, dtype=np.float64)
    tau = np.zeros(dim * dim)
    _check(lib.orc_stress_tensor(dim, mu, L.dptr(g), L.dptr(tau)), "stress tensor")
    return tau


def ns_advection_flux(physics, dim, normal, fieldL, fieldR, TL=300.0, TR=300.0):
    n = np.ascontiguousarray(normal, dtype=np.float64)
    a = np.ascontiguousarray(fieldL, dtype=np.float64)
    b = np.ascontiguousarray(fieldR, dtype=np.float64)
    out = np.zeros(2 + dim)
    _check(lib.orc_ns_advection_flux(C.byref(physics), dim, L.dptr(n), L.dptr(a), L.dptr(b), TL, TR, L.dptr(out)), "advection flux")
    return out


def species_advection_flux(physics, dim, normal, fieldL, fieldR, TL=300.0, TR=300.0):
    n = np.ascontiguousarray(normal, dtype=np.float64)
    a = np.ascontiguousarray(fieldL, dtype=np.float64)
    b = np.ascontiguousarray(fieldR, dtype=np.float64)
    out = np.zeros(physics.n_species)
    _check(lib.orc_species_advection_flux(C.byref(physics), dim, L.dptr(n), L.dptr(a), L.dptr(b), TL, TR, L.dptr(out)),
           "species advection flux")
    return out


def lsq_face_weights(mesh):
    d = mesh.desc()
    out = np.zeros((mesh.n_faces, 2, 3))
    _check(lib.orc_lsq_face_weights(C.byref(d), L.dptr(out)), "lsq weights")
    return out


def rhs(mesh, physics: L.PhysicsDesc, U: np.ndarray, aux: np.ndarray | None = None, F: np.ndarray | None = None, threads: int = 1):
    """F += RHS(U) on the CPU; returns (F, aux). aux holds the temperature guess on input."""
    d = mesh.desc()
    nc = U.shape[1]
    dim = mesh.dim
    naux = 1 + dim + physics.n_species
    U = np.ascontiguousarray(U, dtype=np.float64)
    if aux is None:
        aux = np.zeros((mesh.n_cells, naux))
        aux[:, 0] = 300.0
    aux = np.ascontiguousarray(aux, dtype=np.float64)
    if F is None:
        F = np.zeros((mesh.n_cells, nc))
    _check(lib.orc_rhs(C.byref(d), C.byref(physics), L.dptr(U), L.dptr(aux), L.dptr(F), threads), "rhs")
    return F, aux


class OracleRHS:
    """Oracle with its one-time setup done up front (for timing the per-evaluation CPU cost)."""

    def __init__(self, mesh, physics: L.PhysicsDesc):
        self.mesh = mesh
        self.desc = mesh.desc()
        self.physics = physics
        h = lib.orc_create(C.byref(self.desc), C.byref(self.physics))
        if not h:
            raise RuntimeError(f"oracle setup failed: {lib.orc_last_error().decode()}")
        self.h = h

    def __call__(self, U, aux, F, threads=1):
        _check(lib.orc_run(self.h, L.dptr(U), L.dptr(aux), L.dptr(F), threads), "rhs")
        return F

    def close(self):
        if self.h:
            lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
