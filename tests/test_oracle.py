"""CPU tests of the oracle: the FFTW-API shim against scipy/numpy, the numpy
restatement (oracle/scft_oracle.py) against the reference compiled as
oracle/_ref/libscft_ref.so, the harness loop against the reference's own
unmodified driver, and everything against the committed golden fixtures."""
import ctypes
import os

import numpy as np
import pytest
import scipy.fft as sfft

from crysscft_sample_b200 import fields
from oracle import ref
from oracle import scft_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


# ---------------------------------------------------------------- FFTW shim
def _shim():
    L = ctypes.CDLL(ref.SHIM_PATH)
    L.fftw_plan_r2r_3d.restype = ctypes.c_void_p
    L.fftw_plan_r2r_3d.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2 + [ctypes.c_int] * 3 + [ctypes.c_uint]
    L.fftw_plan_many_dft_r2c.restype = ctypes.c_void_p
    L.fftw_plan_many_dft_r2c.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint]
    L.fftw_plan_many_dft_c2r.restype = ctypes.c_void_p
    L.fftw_plan_many_dft_c2r.argtypes = L.fftw_plan_many_dft_r2c.argtypes
    L.fftw_execute.argtypes = [ctypes.c_void_p]
    L.fftw_destroy_plan.argtypes = [ctypes.c_void_p]
    return L


@needs_ref
@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 12, 10), (6, 10, 14), (5, 7, 9)])
@pytest.mark.parametrize("kinds,scipy_type", [((5, 5, 5), 2), ((4, 4, 4), 3)])  # REDFT10 / REDFT01
def test_shim_r2r_matches_scipy(shape, kinds, scipy_type):
    L = _shim()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape)
    y = np.zeros(shape)
    p = L.fftw_plan_r2r_3d(*shape, x.ctypes.data, y.ctypes.data, *kinds, 0)
    L.fftw_execute(p)
    L.fftw_destroy_plan(p)
    want = sfft.dctn(x, type=scipy_type)
    assert np.abs(y - want).max() < 1e-12 * np.abs(want).max()


@needs_ref
@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 6, 10), (9, 5, 6), (16, 16, 32)])
def test_shim_r2c_c2r_match_numpy(shape):
    L = _shim()
    rng = np.random.default_rng(2)
    x = rng.standard_normal(shape)
    h = shape[2] // 2 + 1
    spec = np.zeros(shape[:2] + (h,), dtype=np.complex128)
    n = (ctypes.c_int * 3)(*shape)
    p = L.fftw_plan_many_dft_r2c(3, n, 1, x.ctypes.data, None, 1, 0, spec.ctypes.data, None, 1, 0, 0)
    L.fftw_execute(p)
    assert np.abs(spec - np.fft.rfftn(x)).max() < 1e-12 * np.abs(spec).max()
    back = np.zeros(shape)
    p2 = L.fftw_plan_many_dft_c2r(3, n, 1, spec.ctypes.data, None, 1, 0, back.ctypes.data, None, 1, 0, 0)
    L.fftw_execute(p2)
    assert np.abs(back / np.prod(shape) - x).max() < 1e-13


# ------------------------------------------------ restatement vs reference
@needs_ref
@pytest.mark.parametrize("kind,N,L", [
    ("PMMM", (32, 32, 32), (4.2, 4.2, 4.2)),
    ("PMMM", (16, 48, 32), (5.0, 5.0, 5.0)),
    ("3M", (32, 16, 48), (4.2, 3.7, 5.1)),
    ("P1", (24, 16, 8), (4.2, 3.7, 5.1)),
])
def test_restatement_triplet_matches_reference(kind, N, L):
    R = ref.RefSolver(kind, N)
    R.set_cell_para(L)
    R.set_contour_step(0.01)
    S = O.OracleSolver(kind, N)
    S.set_cell_para(L)
    S.set_contour_step(0.01)
    q = np.random.default_rng(3).standard_normal(R.space_size_phy)
    assert np.abs(R.diffusion(q) - S.diffusion(q).ravel()).max() < 2e-15


@needs_ref
@pytest.mark.parametrize("kind", ["PMMM", "3M", "P1"])
def test_restatement_iterations_match_reference(kind):
    N, L = (16, 16, 16), 4.0
    wA, wB = fields.seed_fields(N, L)
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    want = ref.RefSolver(kind, N).scft_run(0.3, 0.02, 15.0, (L, L, L), 0.1, 4, a, b)
    got = O.scft_iterations(O.OracleSolver(kind, N), 0.3, 0.02, 15.0, (L, L, L), 0.1, 4, a, b)
    assert np.abs(got["F"] - want["F"]).max() < 1e-13
    assert np.abs(got["phiA"].ravel() - want["phiA"]).max() < 1e-14


@needs_ref
def test_harness_loop_matches_unmodified_driver(tmp_path):
    """ref_scft_run repeats the driver loop; the driver's own printout pins it (10 digits)."""
    N, L = (16, 16, 16), 4.2
    wA, wB = fields.seed_fields(N, L)
    a, b = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)
    R = ref.RefSolver("PMMM", N)
    log = R.run_driver(0.25, 0.01, 20.0, (L, L, L), 0.1, 21, a, b, str(tmp_path / "SolverPmmmDCT"))
    rows = ref.parse_driver_log(log)
    assert [r[0] for r in rows] == [0, 10, 20]
    run = ref.RefSolver("PMMM", N).scft_run(0.25, 0.01, 20.0, (L, L, L), 0.1, 21, a, b)
    for it, F, mi in rows:
        assert abs(run["F"][it] - F) <= 1e-9 * abs(F)
        assert abs(run["maxinc"][it] - mi) <= 1e-9 * abs(mi)
    assert os.path.exists(str(tmp_path / "SolverPmmmDCT_output.txt"))


# ------------------------------------------------------------ golden fixtures
def test_restatement_matches_golden_triplets():
    g = np.load(os.path.join(GOLDEN, "triplets.npz"))
    for kind, N in (("PMMM", (32, 32, 32)), ("3M", (32, 16, 48)), ("P1", (16, 24, 8))):
        k = f"{kind}_{N[0]}x{N[1]}x{N[2]}"
        S = O.OracleSolver(kind, N)
        S.set_cell_para(tuple(g[k + "_cell"]))
        S.set_contour_step(float(g[k + "_ds"]))
        assert np.abs(S.diffusion(g[k + "_in"]).ravel() - g[k + "_out"]).max() < 2e-15


def test_restatement_matches_golden_contours():
    g = np.load(os.path.join(GOLDEN, "contour.npz"))
    for kind in ("PMMM", "3M", "P1"):
        S = O.OracleSolver(kind, (16, 16, 16))
        S.set_cell_para((4.2, 4.2, 4.2))
        S.set_contour_step(0.01)
        wds = g[kind + "_wds"].reshape(S.grid_phy)
        M = S.space_size_phy
        ones = np.ones(S.grid_phy)
        for d, key in ((1, "_fwd"), (-1, "_bwd")):
            got = O.solve_diffusion_equation(S, ones, wds, 10, d).reshape(11, M)
            assert np.abs(got - g[kind + key]).max() < 1e-14


def test_restatement_matches_golden_scft_cfg0():
    """First 15 of the 100 golden iterations (the full run is the GPU test's job)."""
    g = np.load(os.path.join(GOLDEN, "scft_cfg0.npz"))
    N = (32, 32, 32)
    for kind in ("PMMM", "3M"):
        out = O.scft_iterations(O.OracleSolver(kind, N), 0.25, 0.01, 20.0, (4.2,) * 3, 0.1, 15,
                                fields.to_physical(kind, g["wA_full"]), fields.to_physical(kind, g["wB_full"]))
        assert np.all(np.abs(out["F"] - g[kind + "_F"][:15]) <= 1e-12 * np.abs(g[kind + "_F"][:15]))


def test_golden_cross_solver_consistency():
    """The reference's only self-check (Readme.md:30-72): the three solvers agree."""
    g = np.load(os.path.join(GOLDEN, "scft_cfg0.npz"))
    for kind in ("3M", "P1"):
        assert np.abs(g[kind + "_F"] - g["PMMM_F"]).max() < 1e-12 * np.abs(g["PMMM_F"]).max()
        assert np.abs(g[kind + "_maxinc"] - g["PMMM_maxinc"]).max() < 1e-11


def test_golden_seed_fields_reproducible():
    g = np.load(os.path.join(GOLDEN, "scft_cfg0.npz"))
    wA, wB = fields.seed_fields((32, 32, 32), 4.2, "BCC")
    assert np.array_equal(wA, g["wA_full"]) and np.array_equal(wB, g["wB_full"])


# ------------------------------------------- Kronecker form of the triplet
def _axis_ops(kind, N, L, ds):
    PI = np.pi
    g = lambda k, Lc: np.exp(-ds * (2 * PI * k / Lc) ** 2)  # noqa: E731

    def circ(Nn, Lc):
        k = np.arange(Nn)
        return (g(np.minimum(k, Nn - k), Lc)[None, :] * np.cos(2 * PI * np.outer(k, k) / Nn)).sum(1) / Nn

    ops = []
    for d in range(3):
        if kind == "PMMM":
            n = N[d] // 2
            j = np.arange(n)
            c = np.where(j == 0, 1.0, 2.0)
            C = np.cos(PI * np.outer(j, 2 * j + 1) / (2 * n))  # C[k][j]
            ops.append((C.T * (c * g(j, L[0]))) @ C / n)
        elif kind == "P1":
            c = circ(N[d], L[d])
            i = np.arange(N[d])
            ops.append(c[(i[:, None] - i[None, :]) % N[d]])
        else:
            c = circ(N[d], L[d])
            i = np.arange(N[d] // 2)
            ops.append(c[(2 * i[:, None] - 2 * i[None, :]) % N[d]]
                       + c[(2 * i[:, None] + 2 * i[None, :] + 1 - N[d]) % N[d]])
    return ops


@needs_ref
@pytest.mark.parametrize("kind,N,L", [("PMMM", (32, 16, 48), (4.2,) * 3), ("P1", (12, 16, 8), (4.2, 3.7, 5.1)),
                                      ("3M", (24, 16, 32), (4.2, 3.7, 5.1))])
def test_triplet_is_kronecker_of_axis_operators(kind, N, L):
    """The GPU design's premise: every reference triplet equals A_x (x) A_y (x) A_z."""
    R = ref.RefSolver(kind, N)
    R.set_cell_para(L)
    R.set_contour_step(0.01)
    shp = R.grid_size_phy
    q = np.random.default_rng(4).standard_normal(shp)
    Ax, Ay, Az = _axis_ops(kind, N, L, 0.01)
    got = np.einsum("ia,jb,kc,abc->ijk", Ax, Ay, Az, q)
    assert np.abs(got.ravel() - R.diffusion(q.ravel())).max() < 1e-13


@needs_ref
def test_reference_grid_rules_refused_without_exit():
    with pytest.raises(ValueError):
        ref.RefSolver("PMMM", (32, 32, 24))  # (Nz/2) % 8 != 0: the reference would exit(1)
    with pytest.raises(ValueError):
        ref.RefSolver("P1", (16, 16, 12))
