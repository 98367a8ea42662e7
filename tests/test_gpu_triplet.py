"""GPU triplet parity: each GPU solver against the reference solver compiled as the
CPU oracle (oracle/_ref), on the same seeded inputs, through the C ABI."""
import numpy as np
import pytest

from oracle import ref
from crysscft_sample_b200 import solvers as S

pytestmark = pytest.mark.gpu

TOL_TRIPLET = 1e-13  # FP64 max-abs on O(1) data (FFT vs dense-operator rounding)

CASES = [
    ("PMMM", (32, 32, 32), (4.2, 4.2, 4.2), 0.01),
    ("PMMM", (128, 128, 128), (4.2, 4.2, 4.2), 0.005),
    ("PMMM", (16, 48, 32), (5.0, 5.0, 5.0), 0.01),
    ("3M", (32, 32, 32), (4.2, 4.2, 4.2), 0.01),
    ("3M", (32, 16, 48), (4.2, 3.7, 5.1), 0.01),
    ("3M", (128, 128, 128), (4.2, 4.2, 4.2), 0.005),
    ("P1", (32, 32, 32), (4.2, 4.2, 4.2), 0.01),
    ("P1", (24, 16, 40), (4.2, 3.7, 5.1), 0.01),
    ("P1", (64, 64, 64), (5.0, 5.0, 5.0), 0.01),
    # large cubic grids: the FP64 tensor-core axis passes (even/odd and full operators)
    ("PMMM", (256, 256, 256), (4.2, 4.2, 4.2), 0.005),
    ("3M", (256, 256, 256), (4.2, 4.2, 4.2), 0.005),
    ("P1", (128, 128, 128), (4.2, 4.2, 4.2), 0.005),
    ("PMMM", (192, 192, 192), (5.0, 5.0, 5.0), 0.01),
]


@pytest.mark.parametrize("kind,N,L,ds", CASES)
def test_triplet_matches_reference(gpu, kind, N, L, ds):
    rng = np.random.default_rng(hash((kind, N)) % 2**32)
    R = ref.RefSolver(kind, N)
    R.set_cell_para(L)
    R.set_contour_step(ds)
    G = S.make_solver(kind, N)
    G.set_cell_para(L)
    G.set_contour_step(ds)
    assert G.get_grid_size_phy() == R.grid_size_phy
    q = rng.standard_normal(R.space_size_phy)
    want = R.diffusion(q)
    io = G.get_iomat_for_diffusion()
    io[:] = q
    G.diffusion()
    got = io.copy()
    assert np.abs(got - want).max() < TOL_TRIPLET


@pytest.mark.parametrize("kind,N", [("PMMM", (32, 32, 32)), ("3M", (32, 32, 32)), ("P1", (32, 32, 32)),
                                    ("PMMM", (256, 256, 256)), ("P1", (128, 128, 128))])
def test_propagate_matches_reference(gpu, kind, N):
    from crysscft_sample_b200 import fields, scft

    L = 4.2
    ds = 0.01
    wA, _ = fields.seed_fields(N, L)
    w = fields.to_physical(kind, wA).ravel()
    wds = np.exp(-ds / 2 * w)
    R = ref.RefSolver(kind, N)
    R.set_cell_para((L, L, L))
    R.set_contour_step(ds)
    G = S.make_solver(kind, N)
    G.set_cell_para((L, L, L))
    G.set_contour_step(ds)
    M = R.space_size_phy
    init = np.ones(M)
    ns = 25 if N[0] <= 64 else 4
    for direction in (1, -1):
        want = R.solve_diffusion_equation(init, wds, ns, direction)
        got = np.zeros((ns + 1) * M)
        scft.solve_diffusion_equation(got, init, wds, G, ns, direction)
        assert np.abs(got.reshape(ns + 1, M) - want).max() < 1e-12
