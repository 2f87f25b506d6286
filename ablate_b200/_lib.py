"""ctypes binding of ``include/ablate_fv.h`` (the in-tree ``lib/libablate_fv.so``).

Loading fails loudly: if the shared library is missing or lacks a declared symbol, an ImportError
is raised -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libablate_fv.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "ablate_fv.h"

# ---- constants mirrored from the header ------------------------------------------------------
OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_CUDA = -2
ERR_NAN = -3
ERR_EOS_NOT_CONVERGED = -4
ERR_RIEMANN_NOT_CONVERGED = -5
ERR_OUT_OF_MEMORY = -6
ERR_UNSUPPORTED = -7
ERR_NO_DEVICE = -8

FLUX_OFF, FLUX_AVERAGE, FLUX_AUSM, FLUX_AUSMPUP, FLUX_RIEMANN = range(5)
DIR_NA, DIR_LEFT, DIR_RIGHT = 0, 1, 2
EOS_PERFECT_GAS, EOS_NASA7 = 0, 1
(PROP_PRESSURE, PROP_TEMPERATURE, PROP_INTERNAL_SENSIBLE_ENERGY, PROP_SENSIBLE_ENTHALPY, PROP_CV, PROP_CP,
 PROP_SPEED_OF_SOUND, PROP_SPECIES_SENSIBLE_ENTHALPY, PROP_DENSITY) = range(9)
TRANSPORT_NONE, TRANSPORT_CONSTANT, TRANSPORT_SUTHERLAND, TRANSPORT_CONSTANT_LEWIS = range(4)
RECON_UPWIND, RECON_LEASTSQUARES = 0, 1
LIMITER_NONE, LIMITER_ZERO, LIMITER_MINMOD, LIMITER_VANLEER, LIMITER_VANALBADA, LIMITER_SIN = range(6)
CELL_OWNED, CELL_BOUNDARY, CELL_HALO, CELL_HALO_OUTER = range(4)
PRECISION_FP64, PRECISION_MIXED = 0, 1
BC_OUTFLOW, BC_DIRICHLET, BC_SLIP_WALL, BC_NOSLIP_WALL = range(4)
BC_MAX_COMPONENTS = 16
JVP_EXACT, JVP_FROZEN_LIMITER = 0, 1
STEP_EULER, STEP_SSPRK3 = 0, 1
RHS_OVERWRITE = 0x100
RHS_PHASE_INTERIOR, RHS_PHASE_REST = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class BoundaryCondition(C.Structure):
    _fields_ = [("kind", C.c_int32), ("enforce_at_face", C.c_int32), ("value", C.c_double * BC_MAX_COMPONENTS)]


class MeshDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("n_cells", C.c_int32), ("n_faces", C.c_int32),
        ("face_cells", _ip), ("face_normal", _dp), ("face_centroid", _dp),
        ("cell_centroid", _dp), ("cell_volume", _dp), ("cell_kind", _u8p), ("face_shift", _dp),
    ]


class PhysicsDesc(C.Structure):
    _fields_ = [
        ("eos", C.c_int32), ("gamma", C.c_double), ("r_gas", C.c_double), ("n_species", C.c_int32),
        ("nasa7", _dp), ("mw", _dp),
        ("flux", C.c_int32), ("ausmpup_minf", C.c_double), ("pgs_alpha", C.c_double),
        ("reconstruction", C.c_int32), ("limiter", C.c_int32), ("max_lim_grad", C.c_double),
        ("transport", C.c_int32), ("k", C.c_double), ("mu", C.c_double), ("diff", C.c_double),
        ("advection", C.c_int32), ("diffusion", C.c_int32), ("species_advection", C.c_int32), ("species_diffusion", C.c_int32),
        ("species_diff", _dp), ("species_advection_compact", C.c_int32),
    ]


# every entry point declared in the header: name -> (restype, argtypes)
SIGNATURES = {
    "abl_last_error_string": (C.c_char_p, []),
    "abl_version": (C.c_int, []),
    "abl_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "abl_fv_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(PhysicsDesc), C.c_int, C.POINTER(C.c_void_p)]),
    "abl_fv_destroy": (C.c_int, [C.c_void_p]),
    "abl_fv_sizes": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _ip]),
    "abl_fv_record_classes": (C.c_int, [C.c_void_p, _ip, _ip]),
    "abl_fv_fused_info": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _ip]),
    "abl_fv_rhs": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "abl_fv_rhs_host": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp, C.c_int]),
    "abl_fv_rhs_phase": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "abl_fv_jvp": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_jvp_host": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp, _dp, _dp]),
    "abl_fv_vjp": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_vjp_host": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp, _dp]),
    "abl_fv_update_aux": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_update_aux_host": (C.c_int, [C.c_void_p, _dp]),
    "abl_fv_get_aux": (C.c_int, [C.c_void_p, _dp]),
    "abl_fv_set_aux": (C.c_int, [C.c_void_p, _dp]),
    "abl_fv_status": (C.c_int, [C.c_void_p]),
    "abl_fv_launch_count": (C.c_int, [C.c_void_p, C.c_int, _ip]),
    "abl_fv_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "abl_fv_profile_read": (C.c_int, [C.c_void_p, _ip, C.POINTER(C.c_float), C.c_char_p]),
    "abl_flux_calculator_batch": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int64] + [_dp] * 10 + [_ip]),
    "abl_eos_batch": (C.c_int, [C.POINTER(PhysicsDesc), C.c_int, C.c_int, C.c_int64, _dp, _dp, _dp]),
    "abl_eos_batch_noalloc": (C.c_int, [C.POINTER(PhysicsDesc), C.c_int, C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "abl_fv_set_boundary": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, _ip]),
    "abl_fv_fill_ghosts": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "abl_fv_fill_ghosts_jvp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_set_jvp_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "abl_fv_download_owned": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "abl_fv_step_cfl": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "abl_fv_upload_owned": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "abl_fv_fill_ghosts_vjp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_set_pressure_functional": (C.c_int, [C.c_void_p, C.c_int32, _ip, C.c_void_p]),
    "abl_fv_pressure_functional": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p, C.c_void_p]),
    "abl_fv_cfl_dt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_double), C.c_void_p]),
    "abl_fv_normalize_species": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "abl_fv_rk_stage": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "abl_fv_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "abl_rows_gather": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "abl_rows_scatter": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "abl_rows_scatter_add": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
}


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ablate_b200/build.py` "
                          "(the B200 backend has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        try:
            fn = getattr(lib, name)
        except AttributeError as e:
            raise ImportError(f"{LIB_PATH} does not export {name}") from e
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def get():
    """The loaded library, mapped on the first call (importing the package maps nothing, so code that
    only builds meshes, workloads or physics descriptors -- the oracle's CPU runs among them -- never
    loads the CUDA library)."""
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def __getattr__(name):
    # `_lib.lib` loads the library on first use
    if name == "lib":
        return get()
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


class AblateError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc: int, what: str = ""):
    if rc != OK:
        msg = get().abl_last_error_string().decode(errors="replace")
        raise AblateError(rc, f"{what}: {msg}" if what else msg)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "expected a C-contiguous float64 array"
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def u8ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_u8p)


def device_count() -> int:
    n = C.c_int(0)
    rc = get().abl_device_count(C.byref(n))
    return n.value if rc == OK else 0
