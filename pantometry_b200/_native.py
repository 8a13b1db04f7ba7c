"""ctypes binding of libpantometry_b200.so (the C ABI in include/pantometry_gpu.h).

Loading fails loudly: if the library is missing or cannot be loaded, importing the domain
classes raises. There is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpantometry_b200.so")

PM_OK, PM_NO_DEVICE, PM_UNSUPPORTED, PM_VIOLATION = 0, 1, 2, 3
PM_DEVICE_TIMEOUT, PM_BAD_ARG, PM_CUDA_ERROR, PM_OUT_OF_MEMORY = 4, 5, 6, 7
PM_PLAIN_F64, PM_FIELDS_F32 = 0, 1


class Violation(C.Structure):
    """`pm_violation`: a `Violation` (crates/pantometry-core/src/conserved.rs:128-143)."""

    _fields_ = [
        ("quantity", C.c_char * 32),
        ("site", C.c_char * 96),
        ("before", C.c_double),
        ("after", C.c_double),
        ("scale", C.c_double),
        ("tolerance", C.c_double),
        ("step", C.c_longlong),
    ]

    def as_dict(self):
        return {
            "quantity": self.quantity.decode(),
            "site": self.site.decode(),
            "before": self.before,
            "after": self.after,
            "scale": self.scale,
            "tolerance": self.tolerance,
            "step": self.step,
        }


class Ledger(C.Structure):
    _fields_ = [
        ("total", C.c_double),
        ("scale", C.c_double),
        ("parts", C.c_double * 4),
        ("n_parts", C.c_int),
        ("steps", C.c_longlong),
    ]


class Substance(C.Structure):
    _fields_ = [
        ("density", C.c_double),
        ("conductivity", C.c_double),
        ("specific_heat", C.c_double),
        ("emissivity", C.c_double),
        ("thermal", C.c_int),
    ]


class HeatDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double),
        ("substance", Substance),
        ("initial_kelvin", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class HallDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("width", C.c_double), ("height", C.c_double), ("depth", C.c_double),
        ("across", C.c_int),
        ("speed", C.c_double),
        ("density", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class RoomDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("width", C.c_double), ("height", C.c_double),
        ("across", C.c_int),
        ("depth", C.c_double),
        ("density", C.c_double),
        ("speed", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class TubeDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("length", C.c_double),
        ("cells", C.c_int),
        ("area", C.c_double),
        ("density", C.c_double),
        ("speed", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class BarDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("cells", C.c_int),
        ("dx", C.c_double),
        ("area", C.c_double),
        ("substance", Substance),
        ("initial_kelvin", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class CavityDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double),
        ("eps_r", C.c_double), ("mu_r", C.c_double), ("sigma", C.c_double),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class EnsembleGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double),
        ("substance", Substance),
        ("initial_kelvin", C.c_double),
        ("convection_w_per_m2_k", C.c_double),
        ("dt", C.c_double),
    ]


_d, _i, _ll, _sz, _p = C.c_double, C.c_int, C.c_longlong, C.c_size_t, C.c_void_p
_dp = C.POINTER(C.c_double)
_vp = C.POINTER(Violation)
_lp = C.POINTER(Ledger)
_st = C.c_int

SIGNATURES = {
    "pm_status_string": (C.c_char_p, [_st]),
    "pm_last_error": (C.c_char_p, []),
    "pm_device_count": (_st, [C.POINTER(_i)]),
    "pm_version": (C.c_char_p, []),
    # Solid3D
    "pm_heat_create": (_st, [C.POINTER(HeatDesc), C.POINTER(_p)]),
    "pm_heat_fill": (_st, [_p, C.POINTER(Substance), _p, _sz]),
    "pm_heat_losing_from": (_st, [_p, _i, _d, _d, _d]),
    "pm_heat_empty": (_st, [_p, _p, _sz]),
    "pm_heat_dissipating": (_st, [_p, _d, _p, _sz]),
    "pm_heat_generated": (_st, [_p, _dp, _dp]),
    "pm_heat_gaps": (_st, [_p, _p, _p, _p, _sz, C.POINTER(_sz)]),
    "pm_heat_upload": (_st, [_p, _dp, _sz]),
    "pm_heat_download": (_st, [_p, _dp, _sz]),
    "pm_heat_max_stable_dt": (_st, [_p, _dp]),
    "pm_heat_set_tolerance": (_st, [_p, _d]),
    "pm_heat_step": (_st, [_p, _d, _ll, _vp]),
    "pm_heat_ledger": (_st, [_p, _lp]),
    "pm_heat_absorb": (_st, [_p, _d]),
    "pm_heat_checkpoint": (_st, [_p]),
    "pm_heat_restore": (_st, [_p]),
    "pm_heat_sample": (_st, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t]),
    "pm_hall_sample": (_st, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t]),
    "pm_cavity_sample": (_st, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t]),
    "pm_heat_step_kernel": (_st, [_p, C.c_longlong, C.c_char_p, C.c_int, C.POINTER(C.c_longlong)]),
    "pm_heat_set_cells_per_thread": (_st, [_p, _i]),
    "pm_heat_set_stream": (_st, [_p, _p]),
    "pm_heat_set_wait_budget": (_st, [_p, C.c_uint]),
    "pm_heat_destroy": (None, [_p]),
    # Hall
    "pm_hall_create": (_st, [C.POINTER(HallDesc), C.POINTER(_p)]),
    "pm_hall_nodes": (_st, [_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), _dp]),
    "pm_hall_release": (_st, [_p, _dp, _sz]),
    "pm_hall_set_source": (_st, [_p, _ll, _dp, _sz]),
    "pm_hall_set_speed_blocks": (_st, [_p, _i, _dp, _sz]),
    "pm_hall_max_stable_dt": (_st, [_p, _dp]),
    "pm_hall_set_tolerance": (_st, [_p, _d]),
    "pm_hall_step": (_st, [_p, _d, _ll, _vp]),
    "pm_hall_ledger": (_st, [_p, _lp]),
    "pm_hall_download": (_st, [_p, _dp, _dp, _dp, _dp, _dp]),
    "pm_hall_checkpoint": (_st, [_p]),
    "pm_hall_restore": (_st, [_p]),
    "pm_hall_autotune": (_st, [_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pm_hall_set_tile": (_st, [_p, C.c_int, C.c_int]),
    "pm_hall_tile": (_st, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pm_hall_set_stream": (_st, [_p, _p]),
    "pm_hall_destroy": (None, [_p]),
    "pm_room_create": (_st, [C.POINTER(RoomDesc), C.POINTER(_p)]),
    "pm_room_cells": (_st, [_p, C.POINTER(_i), C.POINTER(_i), _dp]),
    "pm_room_release": (_st, [_p, _dp, _sz]),
    "pm_room_max_stable_dt": (_st, [_p, _dp]),
    "pm_room_set_tolerance": (_st, [_p, _d]),
    "pm_room_step": (_st, [_p, _d, _ll, _vp]),
    "pm_room_ledger": (_st, [_p, _lp]),
    "pm_room_download": (_st, [_p, _dp, _dp, _dp, _dp]),
    "pm_room_sample": (_st, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t]),
    "pm_room_checkpoint": (_st, [_p]),
    "pm_room_restore": (_st, [_p]),
    "pm_room_set_stream": (_st, [_p, _p]),
    "pm_room_destroy": (None, [_p]),
    "pm_tube_create": (_st, [C.POINTER(TubeDesc), C.POINTER(_p)]),
    "pm_tube_cells": (_st, [_p, C.POINTER(_i), _dp]),
    "pm_tube_set_ends": (_st, [_p, _i, _d, _i, _d]),
    "pm_tube_release": (_st, [_p, _dp, _sz]),
    "pm_tube_max_stable_dt": (_st, [_p, _dp]),
    "pm_tube_set_tolerance": (_st, [_p, _d]),
    "pm_tube_step": (_st, [_p, _d, _ll, _vp]),
    "pm_tube_ledger": (_st, [_p, _lp]),
    "pm_tube_download": (_st, [_p, _dp, _dp, _dp]),
    "pm_tube_checkpoint": (_st, [_p]),
    "pm_tube_restore": (_st, [_p]),
    "pm_tube_set_stream": (_st, [_p, _p]),
    "pm_tube_destroy": (None, [_p]),
    "pm_bar_create": (_st, [C.POINTER(BarDesc), C.POINTER(_p)]),
    "pm_bar_upload": (_st, [_p, _dp, _sz]),
    "pm_bar_download": (_st, [_p, _dp, _sz]),
    "pm_bar_sample": (_st, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_size_t]),
    "pm_bar_absorb": (_st, [_p, _d]),
    "pm_bar_deposit": (_st, [_p, _dp, _sz]),
    "pm_bar_max_stable_dt": (_st, [_p, _dp]),
    "pm_bar_set_tolerance": (_st, [_p, _d]),
    "pm_bar_step": (_st, [_p, _d, _ll, _vp]),
    "pm_bar_ledger": (_st, [_p, _lp]),
    "pm_bar_checkpoint": (_st, [_p]),
    "pm_bar_restore": (_st, [_p]),
    "pm_bar_set_stream": (_st, [_p, _p]),
    "pm_bar_destroy": (None, [_p]),
    # Cavity
    "pm_cavity_create": (_st, [C.POINTER(CavityDesc), C.POINTER(_p)]),
    "pm_cavity_fill_cells": (_st, [_p, _dp, _dp, _dp, _sz]),
    "pm_cavity_obstruct": (_st, [_p, _p, _sz]),
    "pm_cavity_set_boundary": (_st, [_p, _i, _i]),
    "pm_cavity_release_mode": (_st, [_p, _i, _i, _d, _d]),
    "pm_cavity_upload": (_st, [_p, _dp, _dp, _dp, _dp, _dp, _dp, _i]),
    "pm_cavity_download": (_st, [_p, _dp, _dp, _dp, _dp, _dp, _dp]),
    "pm_cavity_set_source": (_st, [_p, _ll, _dp, _sz]),
    "pm_cavity_courant_limit": (_st, [_p, _dp]),
    "pm_cavity_set_tolerance": (_st, [_p, _d]),
    "pm_cavity_step": (_st, [_p, _d, _ll, _vp]),
    "pm_cavity_ledger": (_st, [_p, _lp]),
    "pm_cavity_energies": (_st, [_p, _dp, _dp]),
    "pm_cavity_checkpoint": (_st, [_p]),
    "pm_cavity_restore": (_st, [_p]),
    "pm_cavity_autotune": (_st, [_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pm_cavity_set_tile": (_st, [_p, C.c_int, C.c_int]),
    "pm_cavity_tile": (_st, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pm_cavity_set_wall_split": (_st, [_p, C.c_int]),
    "pm_cavity_wall_split": (_st, [_p, C.POINTER(C.c_int)]),
    "pm_cavity_set_stream": (_st, [_p, _p]),
    "pm_cavity_destroy": (None, [_p]),
    # Ensembles
    "pm_ensemble_max_stable_dt": (_st, [C.POINTER(EnsembleGrid), _i, _dp]),
    "pm_ensemble_create": (_st, [C.POINTER(EnsembleGrid), _i, _i, _i, C.POINTER(_p)]),
    "pm_ensemble_upload": (_st, [_p, _dp, _sz]),
    "pm_ensemble_download": (_st, [_p, _dp, _sz]),
    "pm_ensemble_set_tolerance": (_st, [_p, _d]),
    "pm_ensemble_step": (_st, [_p, _ll, _vp]),
    "pm_ensemble_ledgers": (_st, [_p, _lp, _i]),
    "pm_ensemble_set_shape": (_st, [_p, _i, _i]),
    "pm_ensemble_set_brick": (_st, [_p, _i, _i, _i]),
    "pm_ensemble_shape": (_st, [_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "pm_ensemble_autotune": (_st, [_p, _i, C.POINTER(_i), C.POINTER(_i)]),
    "pm_ensemble_set_stream": (_st, [_p, _p]),
    "pm_ensemble_destroy": (None, [_p]),
    # Without allocation
    "pm_hall_step_f32_noalloc": (_st, [_i, _i, _i, _d, _d, _d, _d, _i, _p, _p, _p, _p, _p, _p, _p, _p, _p, _dp]),
}

OPTIONAL_SIGNATURES = {}

_lib = None


class NativeError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{status_name(status)}: {message}")
        self.status = status


def load():
    """Load the library once. Raises if it is missing: there is no fallback path."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python pantometry_b200/build.py`. "
            "pantometry_b200 has no CPU fallback."
        )
    lib = C.CDLL(LIB_PATH)
    for table, required in ((SIGNATURES, True), (OPTIONAL_SIGNATURES, False)):
        for name, (res, args) in table.items():
            if not hasattr(lib, name):
                if required:
                    raise ImportError(f"{LIB_PATH} does not export {name}")
                continue
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    _lib = lib
    return lib


def status_name(status):
    return {0: "PM_OK", 1: "PM_NO_DEVICE", 2: "PM_UNSUPPORTED", 3: "PM_VIOLATION", 4: "PM_DEVICE_TIMEOUT",
            5: "PM_BAD_ARG", 6: "PM_CUDA_ERROR", 7: "PM_OUT_OF_MEMORY"}.get(status, f"status {status}")


def check(status):
    """Raise on anything but PM_OK (PM_VIOLATION is handled by the callers that expect it)."""
    if status != PM_OK:
        raise NativeError(status, load().pm_last_error().decode())
    return status
