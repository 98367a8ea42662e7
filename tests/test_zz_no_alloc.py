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


def test_static_scratch_allocates_nothing_on_a_fresh_solver(gpu):
    # The allocating entry point creates three work fields of space_size_phy doubles on a
    # solver's first triplet (2 MiB each at 64^3 physical); the static one must not.  After
    # a warm-up on another solver (the library's kernels are loaded, the array's address is
    # looked up), a fresh solver's first triplets go through the static entry point only,
    # and the device's free memory must not change.
    import torch

    from crysscft_sample_b200 import _lib, solvers

    L = _lib.load()
    N = (128, 128, 128)  # PMMM: 64^3 physical = SCFT_STATIC_SCRATCH_MAX_POINTS

    def make():
        G = solvers.make_solver("PMMM", N)
        G.set_cell_para((4.2, 4.2, 4.2))
        G.set_contour_step(0.005)
        return G

    warm = make()
    M = warm.get_space_size_phy()
    rng = np.random.default_rng(11)
    q0 = torch.tensor(rng.standard_normal(M), dtype=torch.float64, device="cuda")
    _lib.check(L.scft_solver_diffusion_device_static_scratch(warm.handle, ctypes.c_void_p(q0.data_ptr()), None))
    fresh = make()  # operators are built (and allocated) here, before the measurement
    got = q0.clone()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        _lib.check(L.scft_solver_diffusion_device_static_scratch(fresh.handle, ctypes.c_void_p(got.data_ptr()),
                                                                 None))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    # the same two triplets through the allocating entry point (which allocates now)
    want = q0.clone()
    for _ in range(2):
        _lib.check(L.scft_solver_diffusion_device(warm.handle, ctypes.c_void_p(want.data_ptr()), None))
    torch.cuda.synchronize()
    assert (got - want).abs().max().item() <= TOL
    fresh.close()
    warm.close()


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
