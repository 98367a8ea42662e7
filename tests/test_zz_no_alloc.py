"""The triplet entry point that allocates nothing.

scft_solver_diffusion_device_static_scratch serves callers that cannot allocate
device memory (their device memory belongs to another framework's pool, or they
must avoid the device synchronisation cudaMalloc/cudaFree can cause).  It keeps its
scratch in a static array inside the library.  This test calls it through the C ABI
and checks it against the allocating entry point scft_solver_diffusion_device, on
two calls in a row (the array keeps the previous call's contents, which must not
leak into the next result).  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same tolerance as the triplet parity tests


@pytest.mark.parametrize("kind,N", [("PMMM", (128, 128, 128)), ("3M", (32, 16, 48)), ("P1", (24, 32, 16))])
def test_static_scratch_matches_allocating_entry_point(gpu, kind, N):
    import torch

    from crysscft_sample_b200 import _lib, solvers

    L = _lib.load()
    G = solvers.make_solver(kind, N)
    G.set_cell_para((4.2, 3.9, 5.1))
    G.set_contour_step(0.005)
    M = G.get_space_size_phy()
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    rng = np.random.default_rng(7)
    for call in range(2):
        q = torch.tensor(rng.standard_normal(M), dtype=torch.float64, device="cuda")
        want = q.clone()
        _lib.check(L.scft_solver_diffusion_device(G.handle, ctypes.c_void_p(want.data_ptr()), sp))
        got = q.clone()
        _lib.check(L.scft_solver_diffusion_device_static_scratch(G.handle, ctypes.c_void_p(got.data_ptr()), sp))
        torch.cuda.synchronize()
        err = (got - want).abs().max().item()
        assert err <= TOL, f"call {call}: max |static - allocating| = {err}"
    G.close()


def test_static_scratch_rejects_oversized_grid(gpu):
    import torch

    from crysscft_sample_b200 import _lib, solvers

    L = _lib.load()
    G = solvers.CrysPSSolverP1((128, 128, 128))  # 2^21 points > the static maximum
    G.set_cell_para((4.2, 4.2, 4.2))
    G.set_contour_step(0.01)
    q = torch.zeros(G.get_space_size_phy(), dtype=torch.float64, device="cuda")
    rc = L.scft_solver_diffusion_device_static_scratch(G.handle, ctypes.c_void_p(q.data_ptr()), None)
    assert rc == 1  # SCFT_ERR_INVALID_ARG
    assert b"exceeds the maximum" in L.scft_last_error()
    G.close()
