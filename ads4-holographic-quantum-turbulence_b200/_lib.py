"""ctypes binding of ``libhqt.so`` (the C ABI declared in ``include/hqt.h``).

The library is loaded from this package directory.  There is no fallback:
if the library is missing or does not load, every entry point raises.
"""
from __future__ import annotations

import ctypes
from ctypes import (POINTER, Structure, c_char_p, c_double, c_int, c_int32,
                    c_int64, c_void_p)
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhqt.so"

HQT_OK = 0
HQT_EINVAL = 1
HQT_ENONFINITE = 2
HQT_ECUDA = 3
HQT_ENOMEM = 4
HQT_EUNSUPPORTED = 5

HQT_FP64 = 0
HQT_MIXED = 1

# every function declared in include/hqt.h
EXPORTS = [
    "hqt_abi_version", "hqt_create", "hqt_destroy", "hqt_last_error",
    "hqt_set_stream", "hqt_step", "hqt_step_device", "hqt_rhs_device",
    "hqt_filter_device", "hqt_boundary_order_parameter_device",
    "hqt_winding_device", "hqt_count_vortices", "hqt_count_vortices_device",
    "hqt_profile", "hqt_profile_report", "hqt_config_report",
    "hqt_count_vortices_field_noalloc", "hqt_noalloc_last_error",
    "hqt_energy_spectrum_device", "hqt_boundary_velocity_device", "hqt_observables_device",
    "hqt_find_vortices_device", "hqt_vortex_structure_factor_device",
    "hqt_ensemble_create", "hqt_ensemble_destroy", "hqt_ensemble_set_stream",
    "hqt_ensemble_last_error", "hqt_ensemble_step_device",
]


class hqt_params(Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
                ("Lx", c_double), ("Ly", c_double), ("mu", c_double),
                ("vy", c_double), ("dt", c_double),
                ("remove_winding", c_int32), ("precision", c_int32),
                ("diag_every", c_int32), ("apply_filter", c_int32),
                ("autotune", c_int32)]


class hqt_diag(Structure):
    _fields_ = [("steps_done", c_int64), ("nonfinite_step", c_int64),
                ("last_winding", c_int32), ("n_records", c_int32),
                ("capacity", c_int32), ("reserved", c_int32),
                ("records", POINTER(c_int32)), ("obs", POINTER(c_double))]


class HQTError(RuntimeError):
    """A non-zero status of the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class NonfiniteEvolution(HQTError):
    """The evolved fields became non-finite (the reference stops at its NaN
    guard, ``tevol_driven_cluster.m:182-185``; its smoke test names this
    condition ``hqt:NonfiniteEvolution``)."""


_lib = None


def load() -> ctypes.CDLL:
    """Load ``libhqt.so`` and declare the signatures (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is not built; run `python build.py` in the package "
            "directory (or __graft_entry__.build())")
    lib = ctypes.CDLL(str(LIB_PATH))
    P = POINTER(hqt_params)
    D = POINTER(hqt_diag)
    dp = POINTER(c_double)
    ip = POINTER(c_int32)
    sig = {
        "hqt_abi_version": (c_int, []),
        "hqt_create": (c_int, [P, c_int, POINTER(c_void_p)]),
        "hqt_destroy": (None, [c_void_p]),
        "hqt_last_error": (c_char_p, [c_void_p]),
        "hqt_set_stream": (c_int, [c_void_p, c_void_p]),
        "hqt_step": (c_int, [c_void_p, dp, dp, dp, dp, dp, c_int64, D]),
        "hqt_step_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_int64, D]),
        "hqt_rhs_device": (c_int, [c_void_p] + [c_void_p] * 8),
        "hqt_filter_device": (c_int, [c_void_p, c_void_p, c_void_p, c_int32]),
        "hqt_boundary_order_parameter_device": (c_int, [c_void_p, c_void_p,
                                                        c_void_p]),
        "hqt_winding_device": (c_int, [c_void_p, c_void_p, ip]),
        "hqt_count_vortices": (c_int, [c_void_p, dp, ip, ip, ip]),
        "hqt_count_vortices_device": (c_int, [c_void_p, c_void_p, ip, ip, ip]),
        "hqt_profile": (c_int, [c_void_p, c_int]),
        "hqt_profile_report": (c_int, [c_void_p, ctypes.c_char_p, c_int64]),
        "hqt_config_report": (c_int, [c_void_p, ctypes.c_char_p, c_int64]),
        "hqt_count_vortices_field_noalloc": (c_int, [c_void_p, c_int32, c_int32,
                                                     c_int32, ip, ip, ip, c_void_p]),
        "hqt_noalloc_last_error": (c_char_p, []),
        "hqt_energy_spectrum_device": (c_int, [c_void_p, c_void_p, c_int32, dp, dp, dp,
                                               dp, ip]),
        "hqt_boundary_velocity_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "hqt_observables_device": (c_int, [c_void_p, c_void_p, c_void_p, dp]),
        "hqt_find_vortices_device": (c_int, [c_void_p, c_void_p, c_double, c_int32, c_int32,
                                             dp, dp, ip]),
        "hqt_vortex_structure_factor_device": (c_int, [c_void_p, c_void_p, c_double, c_double,
                                                       c_int32, dp, ip, c_int32, dp, dp, dp,
                                                       ip, dp]),
        "hqt_ensemble_create": (c_int, [POINTER(c_void_p), c_int32, POINTER(c_void_p)]),
        "hqt_ensemble_destroy": (None, [c_void_p]),
        "hqt_ensemble_set_stream": (c_int, [c_void_p, c_void_p]),
        "hqt_ensemble_last_error": (c_char_p, [c_void_p]),
        "hqt_ensemble_step_device": (c_int, [c_void_p] + [POINTER(c_void_p)] * 5
                                     + [c_int64, D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int, ctx=None) -> None:
    """Raise the matching exception for a non-zero status."""
    if code == HQT_OK:
        return
    lib = load()
    msg = lib.hqt_last_error(ctx)
    msg = msg.decode() if msg else ""
    if code == HQT_ENONFINITE:
        raise NonfiniteEvolution(code, msg or "non-finite fields")
    raise HQTError(code, msg)
