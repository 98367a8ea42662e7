"""GPU parity of the 3m solver with mirror translations (src/solver_3m.h:17,
:172-324, src/solver_utilities.h:56-66) against the reference build: the triplet
through every entry point, SCFT iterations, and the physical meaning (P1 on the
symmetric extension) including the stress."""
import ctypes

import numpy as np
import pytest

from crysscft_sample_b200 import _lib, fields, scft, solvers
from oracle import ref

pytestmark = pytest.mark.gpu

N = (32, 24, 32)
L = (4.2, 3.9, 5.0)
GS = [
    (0.5, 0, 0, 0, 0, 0, 0, 0, 0),
    (0, 0, 0, 0, 0, 0.5, 0, 0, 0),
    (0, 0, 0, 0, 1 / 3, 0, 0, 0, 0),
    (0, 0.5, 0, 0.5, 0, 0, 0, 0, 0.5),
    (0.5, 0.5, 0.25, 0.5, 0, 0.5, 0, 0.5, 0.5),
]
CFG = dict(fA=0.25, ds=0.01, xN=20.0, acc=0.1)


def _fields():
    wA, wB = fields.seed_fields(N, L, "BCC")
    rng = np.random.default_rng(21)
    n = tuple(v // 2 for v in N)
    # BCC seed on the even sub-lattice plus noise that no mirror of g = 0 would keep
    return (np.ascontiguousarray(wA[::2, ::2, ::2] + 0.05 * rng.standard_normal(n)),
            np.ascontiguousarray(wB[::2, ::2, ::2] + 0.05 * rng.standard_normal(n)))


@pytest.mark.parametrize("g", GS)
def test_triplet_matches_reference(gpu, g):
    import torch

    R = ref.RefSolver("3M", N, g)
    R.set_cell_para(L)
    R.set_contour_step(0.01)
    G = solvers.CrysPSSolver3m(N, g)
    G.set_cell_para(L)
    G.set_contour_step(0.01)
    q = np.random.default_rng(22).standard_normal(G.get_space_size_phy())
    want = R.diffusion(q)
    scale = np.abs(want).max()
    io = G.get_iomat_for_diffusion()
    io[:] = q
    G.diffusion()
    assert np.abs(io - want).max() < 1e-14 * scale
    t = torch.tensor(q, device="cuda")
    G.diffusion_device(t)  # in place: the library works from a copy of the input
    torch.cuda.synchronize()
    assert np.abs(t.cpu().numpy() - want).max() < 1e-14 * scale
    # a 5-step chain against the reference's step loop (src/crysSCFT_sample.cpp:373-396)
    wds = np.exp(-0.005 * np.random.default_rng(23).standard_normal(q.size))
    chain = R.solve_diffusion_equation(q, wds, 5, 1)
    qd = torch.zeros(6 * q.size, dtype=torch.float64, device="cuda")
    G.propagate_device(qd, torch.tensor(q, device="cuda"), torch.tensor(wds, device="cuda"), 5, 1)
    torch.cuda.synchronize()
    assert np.abs(qd.cpu().numpy().reshape(6, -1) - chain).max() < 1e-14 * np.abs(chain).max()


@pytest.mark.parametrize("g", GS)
def test_iterations_match_reference(gpu, g):
    a, b = _fields()
    want = ref.RefSolver("3M", N, g).scft_run(CFG["fA"], CFG["ds"], CFG["xN"], L, CFG["acc"], 8, a, b)
    G = solvers.CrysPSSolver3m(N, g)
    G.set_cell_para(L)
    run = scft.DiblockSCFT(G, CFG["fA"], CFG["ds"], CFG["xN"], CFG["acc"])
    run.set_fields(a, b)
    got = run.iterate(8)
    got.update(run.get_fields())
    assert np.all(np.abs(got["F"] - want["F"]) <= 1e-10 * np.abs(want["F"]))
    assert np.abs(got["phiA"].ravel() - want["phiA"]).max() < 1e-12
    assert np.abs(got["wB"].ravel() - want["wB"]).max() < 1e-11


@pytest.mark.parametrize("g", [GS[0], GS[4]])
def test_equals_p1_on_the_symmetric_extension(gpu, g):
    """F, phi and the stress of 3m with g equal those of P1 on the extended fields."""
    a, b = _fields()
    out = {}
    for kind in ("3M", "P1"):
        if kind == "3M":
            G = solvers.CrysPSSolver3m(N, g)
            wa, wb = a, b
        else:
            G = solvers.CrysPSSolverP1(N)
            wa, wb = fields.extend_3m(a, N, g), fields.extend_3m(b, N, g)
        G.set_cell_para(L)
        run = scft.DiblockSCFT(G, CFG["fA"], CFG["ds"], CFG["xN"], CFG["acc"])
        run.set_fields(wa, wb)
        h = run.iterate(6)
        phi = run.get_fields()["phiA"]
        if kind == "P1":
            phi = phi.reshape(N)[::2, ::2, ::2]
        out[kind] = (h["F"], phi.ravel(), run.stress()["dlnQ_dL"])
    (F3, p3, s3), (F1, p1, s1) = out["3M"], out["P1"]
    assert np.all(np.abs(F3 - F1) <= 1e-12 * np.abs(F1))
    assert np.abs(p3 - p1).max() < 1e-12
    assert np.allclose(s3, s1, rtol=1e-9, atol=1e-13)


def test_fp32_multi_term(gpu):
    """The FP32 form on a multi-term operator (per-axis kernels) tracks FP64."""
    a, b = _fields()
    F = {}
    for prec in ("fp64", "fp32"):
        G = solvers.CrysPSSolver3m(N, GS[4])
        G.set_cell_para(L)
        run = scft.DiblockSCFT(G, CFG["fA"], CFG["ds"], CFG["xN"], CFG["acc"])
        run.set_precision(prec)
        run.set_fields(a, b)
        F[prec] = run.iterate(5)["F"]
    assert np.all(np.abs(F["fp32"] - F["fp64"]) <= 3e-5 * np.abs(F["fp64"]))


def test_static_scratch_refuses_multi_term(gpu):
    import torch

    G = solvers.CrysPSSolver3m(N, GS[0])
    G.set_cell_para(L)
    G.set_contour_step(0.01)
    q = torch.ones(G.get_space_size_phy(), dtype=torch.float64, device="cuda")
    rc = _lib.load().scft_solver_diffusion_device_static_scratch(G.handle, ctypes.c_void_p(q.data_ptr()), None)
    assert rc == 8  # SCFT_ERR_UNSUPPORTED
