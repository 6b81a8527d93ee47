"""ctypes binding of libicar_adv.so (the C ABI declared in include/icar_adv.h).

The shared library is built in-tree (hicar_b200/build.py).  Loading fails
loudly when it is missing: there is no CPU fallback for the advection step.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libicar_adv.so"

MAX_SPECIES = 32

# status codes (icar_adv_status)
OK, BAD_ARG, OOM, CFL_VIOLATION, NAN_INPUT, TIMEOUT, CUDA_ERROR, NOT_READY, OVER_BUDGET, PHYSICS_STOP = range(10)
STATUS_NAMES = {
    0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "CFL_VIOLATION", 4: "NAN_INPUT", 5: "TIMEOUT",
    6: "CUDA_ERROR", 7: "NOT_READY", 8: "OVER_BUDGET", 9: "PHYSICS_STOP",
}

# field ids (kVARS numbering, src/constants/icar_constants.f90)
F_U, F_V, F_W = 1, 2, 3
F_THETA, F_QV, F_QC, F_NC, F_QI, F_NI, F_QR, F_NR, F_QS, F_NS, F_QG, F_NG = 7, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19
F_DENSITY, F_DZ_INTERFACE = 39, 43
F_PRESSURE, F_EXNER, F_DZ_MASS = 5, 37, 42
F_JACOBIAN, F_JACOBIAN_U, F_JACOBIAN_V, F_JACOBIAN_W, F_ADVECTION_DZ, F_RELAX_FILTER = 1001, 1002, 1003, 1004, 1005, 1006
F_FORCING_BASE, F_DQDT_BASE = 2000, 3000

SPECIES_IDS = {
    "theta": F_THETA, "qv": F_QV, "qc": F_QC, "nc": F_NC, "qi": F_QI, "ni": F_NI, "qr": F_QR,
    "nr": F_NR, "qs": F_QS, "ns": F_NS, "qg": F_QG, "ng": F_NG,
}
SPECIES_NAMES = {v: k for k, v in SPECIES_IDS.items()}


class Desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_float),
        ("n_species", C.c_int32),
        ("species", C.c_int32 * MAX_SPECIES),
        ("north_boundary", C.c_int32), ("south_boundary", C.c_int32),
        ("east_boundary", C.c_int32), ("west_boundary", C.c_int32),
        ("device", C.c_int32),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("advection", C.c_int32), ("mpdata_fct", C.c_int32), ("mpdata_order", C.c_int32),
        ("flux_corr", C.c_int32), ("h_order", C.c_int32), ("v_order", C.c_int32),
        ("rk3", C.c_int32), ("advect_density", C.c_int32), ("debug", C.c_int32),
        ("boundary_buffer", C.c_int32),
    ]


class NoallocArgs(C.Structure):
    """icar_adv_noalloc_args: device pointers in the pitched layout."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_float), ("dt", C.c_float),
        ("mpdata_fct", C.c_int32), ("advect_density", C.c_int32), ("n_species", C.c_int32),
        ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("density", C.c_void_p),
        ("jacobian", C.c_void_p), ("jacobian_u", C.c_void_p), ("jacobian_v", C.c_void_p),
        ("jacobian_w", C.c_void_p), ("advection_dz", C.c_void_p),
        ("q_in", C.c_void_p * MAX_SPECIES), ("q_out", C.c_void_p * MAX_SPECIES),
        ("stream", C.c_void_p),
    ]


# every exported entry point, with argument and result types
_PROTOS = {
    "icar_adv_abi_version": (C.c_int, []),
    "icar_adv_default_opts": (C.c_int, [C.POINTER(Opts)]),
    "icar_adv_var_request": (C.c_int, [C.POINTER(Opts), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "icar_adv_halo_size": (C.c_int, [C.POINTER(Opts)]),
    "icar_adv_create": (C.c_int, [C.POINTER(Desc), C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "icar_adv_destroy": (C.c_int, [C.c_void_p]),
    "icar_adv_set_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int64)]),
    "icar_adv_get_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int64)]),
    "icar_adv_set_field_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "icar_adv_get_field_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "icar_adv_advect": (C.c_int, [C.c_void_p, C.c_float]),
    "icar_adv_apply_forcing": (C.c_int, [C.c_void_p, C.c_double]),
    "icar_adv_enforce_limits": (C.c_int, [C.c_void_p]),
    "icar_adv_step": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "icar_adv_sync": (C.c_int, [C.c_void_p]),
    "icar_adv_sync_timeout": (C.c_int, [C.c_void_p, C.c_double]),
    "icar_adv_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "icar_adv_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "icar_adv_footprint": (C.c_int, [C.POINTER(Desc), C.POINTER(Opts), C.POINTER(C.c_int64)]),
    "icar_adv_last_error": (C.c_char_p, [C.c_void_p]),
    "icar_adv_set_path": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_profile_read_correction": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "icar_adv_balance_uvw": (C.c_int, [C.c_void_p]),
    "icar_adv_compute_dt": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_float, C.c_int32, C.c_int32,
                                      C.POINTER(C.c_float)]),
    "icar_adv_mp_simple": (C.c_int, [C.c_void_p, C.c_float]),
    "icar_adv_get_precipitation": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "icar_adv_set_precipitation": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "icar_adv_step_host": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "icar_adv_restart_vars": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "icar_adv_download": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_void_p)]),
    "icar_adv_upload": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_void_p)]),
    "icar_adv_set_tile_shape": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_set_species_group": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_batch_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "icar_adv_batch_destroy": (C.c_int, [C.c_void_p]),
    "icar_adv_batch_add": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "icar_adv_batch_remove": (C.c_int, [C.c_void_p, C.c_void_p]),
    "icar_adv_batch_set_dt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "icar_adv_batch_set_tile_shape": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_batch_set_species_group": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_batch_step": (C.c_int, [C.c_void_p]),
    "icar_adv_batch_sync": (C.c_int, [C.c_void_p]),
    "icar_adv_batch_sync_timeout": (C.c_int, [C.c_void_p, C.c_double]),
    "icar_adv_batch_set_path": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "icar_adv_batch_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "icar_adv_batch_profile_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                              C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "icar_adv_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "icar_adv_advect_noalloc": (C.c_int, [C.POINTER(NoallocArgs)]),
    "icar_adv_tile_shapes": (C.c_int, [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "icar_adv_profile_read": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
}

_lib = None


class IcarAdvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libicar_adv.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -m hicar_b200.build` (nvcc, sm_100a). "
            "The advection step has no CPU fallback.")
    lib = C.CDLL(str(p))
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def check(code: int, handle=None) -> None:
    if code != OK:
        lib = load()
        msg = lib.icar_adv_last_error(handle)
        raise IcarAdvError(code, msg.decode() if msg else "")


def f32_ptr(a: np.ndarray):
    assert a.dtype == np.float32
    return a.ctypes.data_as(C.c_void_p)
