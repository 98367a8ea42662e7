"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every
entry point include/crysscft_b200.h declares; host-side argument checks return
the documented status codes (no GPU work is launched here)."""
import ctypes
import os
import re

import pytest

from crysscft_sample_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "crysscft_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(scft_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_plugin_surface():
    names = declared_functions()
    for must in ("scft_solver_create", "scft_solver_destroy", "scft_solver_set_cell_para",
                 "scft_solver_set_contour_step", "scft_solver_diffusion", "scft_solver_get_iomat_for_diffusion",
                 "scft_solver_propagate_device", "scft_diblock_create", "scft_diblock_iterate",
                 "scft_diblock_iterate_host"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.lib_path())
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_python_bindings_cover_the_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_status_strings_and_version():
    L = _lib.load()
    assert L.scft_status_string(0) == b"SCFT_OK"
    assert L.scft_status_string(7) == b"SCFT_ERR_TIMEOUT"
    assert b"sm_100a" in L.scft_version()


def test_argument_errors_are_status_codes():
    L = _lib.load()
    h = ctypes.c_void_p()
    grid = (ctypes.c_size_t * 3)(32, 32, 32)
    assert L.scft_solver_create(5, grid, None, 0, -1, ctypes.byref(h)) == 1  # bad kind
    assert L.scft_solver_create(0, grid, None, 7, -1, ctypes.byref(h)) == 1  # bad precision
    odd = (ctypes.c_size_t * 3)(31, 32, 32)
    assert L.scft_solver_create(2, odd, None, 0, -1, ctypes.byref(h)) == 2  # PMMM needs even sizes
    assert L.scft_solver_destroy(None) == 0
    assert L.scft_diblock_destroy(None) == 0
    assert L.scft_solver_diffusion(None) == 1


def test_no_gpu_is_reported_not_emulated():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.load()
    h = ctypes.c_void_p()
    grid = (ctypes.c_size_t * 3)(32, 32, 32)
    assert L.scft_solver_create(2, grid, None, 0, -1, ctypes.byref(h)) == 9  # SCFT_ERR_NO_DEVICE
    assert h.value is None
