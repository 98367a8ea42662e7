"""Loader of the in-tree CUDA library (ctypes).  There is no CPU fallback: if the
library cannot be built or loaded, every entry point raises."""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_szp = ctypes.POINTER(ctypes.c_size_t)
_ip = ctypes.POINTER(ctypes.c_int)

SCFT_OK = 0
STATUS = {
    0: "SCFT_OK", 1: "SCFT_ERR_INVALID_ARG", 2: "SCFT_ERR_BAD_GRID", 3: "SCFT_ERR_CUDA",
    4: "SCFT_ERR_ALLOC", 5: "SCFT_ERR_NOT_READY", 6: "SCFT_ERR_NUMERIC", 7: "SCFT_ERR_TIMEOUT",
    8: "SCFT_ERR_UNSUPPORTED", 9: "SCFT_ERR_NO_DEVICE",
}
KIND = {"P1": 0, "3M": 1, "PMMM": 2}
PRECISION = {"fp64": 0, "fp32": 1}

# name -> (restype, argtypes); the exported C ABI of include/crysscft_b200.h
SIGNATURES = {
    "scft_last_error": (ctypes.c_char_p, []),
    "scft_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "scft_version": (ctypes.c_char_p, []),
    "scft_solver_create": (ctypes.c_int, [ctypes.c_int, _szp, _dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "scft_solver_destroy": (ctypes.c_int, [_vp]),
    "scft_operator_terms": (ctypes.c_int, [ctypes.c_int, _szp, _dp, _dp, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_size_t), _dp, ctypes.c_size_t]),
    "scft_solver_set_cell_para": (ctypes.c_int, [_vp, _dp]),
    "scft_solver_set_contour_step": (ctypes.c_int, [_vp, ctypes.c_double]),
    "scft_solver_get_grid_size_log": (ctypes.c_int, [_vp, _szp]),
    "scft_solver_get_grid_size_phy": (ctypes.c_int, [_vp, _szp]),
    "scft_solver_get_space_size_phy": (ctypes.c_int, [_vp, _szp]),
    "scft_solver_get_cell_para": (ctypes.c_int, [_vp, _dp]),
    "scft_solver_get_ds": (ctypes.c_int, [_vp, _dp]),
    "scft_solver_get_iomat_for_diffusion": (ctypes.c_int, [_vp, ctypes.POINTER(_dp)]),
    "scft_solver_diffusion": (ctypes.c_int, [_vp]),
    "scft_solver_diffusion_device": (ctypes.c_int, [_vp, _vp, _vp]),
    "scft_solver_propagate_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, _sz, ctypes.c_int, _vp]),
    "scft_solver_propagate": (ctypes.c_int, [_vp, _dp, _dp, _dp, _sz, ctypes.c_int]),
    "scft_diblock_create": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.POINTER(_vp)]),
    "scft_diblock_destroy": (ctypes.c_int, [_vp]),
    "scft_diblock_get_contour_counts": (ctypes.c_int, [_vp, _szp, _szp]),
    "scft_diblock_get_solver": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "scft_diblock_set_fields": (ctypes.c_int, [_vp, _dp, _dp]),
    "scft_diblock_get_fields": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "scft_diblock_device_fields": (ctypes.c_int, [_vp] + [ctypes.POINTER(_vp)] * 4),
    "scft_diblock_iterate": (ctypes.c_int, [_vp, _sz, _dp, _dp, _dp, _dp]),
    "scft_diblock_iterate_host": (ctypes.c_int, [_vp, _dp, _dp, _sz, _dp, _dp, _dp, _dp, _dp, _dp]),
    "scft_diblock_launches_per_iteration": (ctypes.c_int, [_vp, _szp]),
    "scft_diblock_time_phases": (ctypes.c_int, [_vp, _sz, _dp]),
    "scft_solver_set_stream": (ctypes.c_int, [_vp, _vp]),
    "scft_solver_diffusion_device_static_scratch": (ctypes.c_int, [_vp, _vp, _vp]),
    "scft_measure_fp64_peak": (ctypes.c_int, [ctypes.c_int, _dp, _dp]),
    "scft_diblock_set_precision": (ctypes.c_int, [_vp, ctypes.c_int]),
    "scft_diblock_get_contour": (ctypes.c_int, [_vp, ctypes.c_int, _sz, _dp]),
    "scft_diblock_stress": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "scft_solver_set_pmmm_anisotropic": (ctypes.c_int, [_vp, ctypes.c_int]),
    "scft_batch_create": (ctypes.c_int, [ctypes.c_int, _sz, _szp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "scft_batch_destroy": (ctypes.c_int, [_vp]),
    "scft_batch_size": (ctypes.c_int, [_vp, _szp]),
    "scft_batch_instance": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(_vp)]),
    "scft_batch_set_fields": (ctypes.c_int, [_vp, _sz, _dp, _dp]),
    "scft_batch_get_fields": (ctypes.c_int, [_vp, _sz, _dp, _dp, _dp, _dp]),
    "scft_batch_iterate": (ctypes.c_int, [_vp, _sz, _dp, _dp]),
    "scft_batch_configure": (ctypes.c_int, [_vp, _sz, ctypes.c_int]),
    "scft_batch_autotune": (ctypes.c_int, [_vp, _sz, _szp, ctypes.POINTER(ctypes.c_int), _dp]),
    "scft_batch_set_team_sizes": (ctypes.c_int, [_vp, _sz, _ip, _ip]),
    "scft_batch_team_plan": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), _szp, _szp, _dp, _dp]),
    "scft_batch_launches_per_iteration": (ctypes.c_int, [_vp, _szp]),
    "scft_team_schedule": (ctypes.c_int, [_sz, _ip, _ip, ctypes.c_int, _sz, _ip, _ip, _ip, _sz, _ip, _ip, _ip,
                                          _ip, _szp, _dp, _dp]),
    "scft_diblock_get_precision": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "scft_diblock_set_mixing": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double]),
    "scft_diblock_get_residuals": (ctypes.c_int, [_vp, _dp, _sz, _szp]),
    "scft_diblock_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "scft_diblock_set_phi_form": (ctypes.c_int, [_vp, ctypes.c_int]),
}

_lib = None


class ScftError(RuntimeError):
    """A non-zero status from the C ABI (the reference prints "ERROR" and exits instead)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load (building first if needed and nvcc is available) the CUDA library."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CRYSSCFT_LIB", _build.LIB)  # alternative build (A/B comparisons)
    if build_if_missing and (not os.path.exists(path) or _build.needs_build()):
        if os.path.exists(_build.NVCC):
            _build.build()
    if not os.path.exists(path):
        raise RuntimeError(f"crysscft_b200 CUDA library missing at {path}; run python -m crysscft_sample_b200.build")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != SCFT_OK:
        msg = load().scft_last_error().decode(errors="replace")
        raise ScftError(status, msg)


def dptr(a):
    return a.ctypes.data_as(_dp)
