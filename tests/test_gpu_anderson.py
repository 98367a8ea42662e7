"""Anderson mixing on the device (scft_diblock_set_mixing; no counterpart in the
reference, which mixes simply, src/crysSCFT_sample.cpp:362-371): per-iteration parity
with the oracle's restatement, convergence to the saddle point, and the precision
form checked at convergence (FP32 iterations, then FP64 Anderson polish, reach the
saddle point of the plain FP64 run)."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers
from oracle import scft_oracle as O

pytestmark = pytest.mark.gpu

N, L, FA, DS, XN = (32, 32, 32), 4.2, 0.25, 0.01, 20.0


def _run(kind="PMMM"):
    wA, wB = fields.seed_fields(N, L)
    G = solvers.make_solver(kind, N)
    G.set_cell_para((L,) * 3)
    run = scft.DiblockSCFT(G, FA, DS, XN, 0.1)
    run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
    return run


@pytest.mark.parametrize("kind", ["PMMM", "P1"])
def test_device_anderson_matches_oracle(gpu, kind):
    run = _run(kind)
    run.iterate(40)  # simple mixing first, as in practice
    f = run.get_fields()
    run.set_fields(f["wA"], f["wB"])
    run.set_mixing("anderson", history=8, beta=0.5)
    got = run.iterate(20)
    res = run.residuals()
    want = O.scft_iterations_anderson(O.OracleSolver(kind, N), FA, DS, XN, (L,) * 3, 8, 0.5, 20, f["wA"], f["wB"])
    # the least-squares solve of every update amplifies rounding differences between the
    # device's and numpy's reductions by the condition number of the normal equations, so
    # the tolerances of the derived quantities are looser than the free energy's
    rel = np.abs(got["F"] - want["F"]) / np.abs(want["F"])
    rres = np.abs(res - want["residual"]) / want["residual"]
    g = run.get_fields()
    dw = np.abs(g["wA"] - want["wA"].ravel()).max()
    dphi = np.abs(g["phiB"] - want["phiB"].ravel()).max()
    msg = f"F {rel.max():.2e} residual {rres.max():.2e} wA {dw:.2e} phiB {dphi:.2e}"
    assert rel.max() < 1e-10, msg
    assert rres.max() < 1e-6, msg
    assert dw < 1e-7 and dphi < 1e-9, msg


def test_simple_mixing_residual_and_switching_back(gpu):
    run = _run()
    f0 = run.get_fields()
    run.iterate(1)
    r_simple = run.residuals()[0]
    want = O.scft_iterations_anderson(O.OracleSolver("PMMM", N), FA, DS, XN, (L,) * 3, 4, 0.5, 1, f0["wA"], f0["wB"])
    assert abs(r_simple - want["residual"][0]) <= 1e-10 * want["residual"][0]
    # Anderson, then back to simple mixing: the reference's update again
    run.set_mixing("anderson", history=4, beta=0.5)
    run.iterate(3)
    run.set_mixing("simple")
    f = run.get_fields()
    got = run.iterate(2)
    want = O.scft_iterations(O.OracleSolver("PMMM", N), FA, DS, XN, (L,) * 3, 0.1, 2, f["wA"], f["wB"])
    assert np.all(np.abs(got["F"] - want["F"]) <= 1e-10 * np.abs(want["F"]))


def test_fp32_then_fp64_anderson_polish_reaches_the_fp64_saddle(gpu):
    def solve(precision):
        run = _run()
        run.set_precision(precision)
        run.iterate(150)
        run.set_precision("fp64")
        run.set_mixing("anderson", history=32, beta=0.5)
        h = run.iterate(200)
        return h, run.residuals()

    h64, r64 = solve("fp64")
    h32, r32 = solve("fp32")
    assert r64[-1] < 1e-10 and r32[-1] < 1e-10
    assert abs(h32["F"][-1] - h64["F"][-1]) <= 1e-10 * abs(h64["F"][-1])
