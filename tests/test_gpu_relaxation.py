"""Variable-cell relaxation of the 128^3 BCC system (PMMM on 64^3, fA = 0.25, chiN = 20,
ds = 0.005) from L = 4.0 Rg to a stress-free cubic cell, in the plain FP64 form and in the
precision form (FP32 triplets to an rms residual of 1e-5 at each cell, then FP64 polish),
with the stress from the adjoint backward pass (scft_diblock_stress).  The reference has
no stress; its cell hook is set_cell_para (src/solver_base.h:16, cubic in PMMM,
src/solver_Pmmm.h:98-104)."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu

N = (128, 128, 128)
PARAMS = dict(fA=0.25, ds=0.005, xN=20.0, acceptance=0.1)


def _start():
    wA, wB = fields.seed_fields(N, 4.0, "BCC")
    return fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)


def _stress_at(G, L, w, precision):
    # stress from one iteration of the given precision on the fields w at cell L
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, PARAMS["fA"], PARAMS["ds"], PARAMS["xN"], PARAMS["acceptance"])
    run.set_fields(*w)
    run.set_precision(precision)
    run.iterate(1)
    g = -float(run.stress()["dlnQ_dL"].sum())
    run.close()
    return g


def test_relaxation_reaches_a_stress_free_cell(gpu):
    a, b = _start()
    G = solvers.make_solver("PMMM", N)
    r64 = scft.relax_cubic_cell(G, PARAMS["fA"], PARAMS["ds"], PARAMS["xN"], PARAMS["acceptance"], a, b, 4.0,
                                tol=1e-8)
    r32 = scft.relax_cubic_cell(G, PARAMS["fA"], PARAMS["ds"], PARAMS["xN"], PARAMS["acceptance"], a, b, 4.0,
                                tol=1e-8, fp32_tol=1e-5)
    for name, r in (("fp64", r64), ("fp32+polish", r32)):
        rows = "; ".join(f"L={h[0]:.9f} F={h[1]:.12f} dF/dL={h[2]:+.3e} it32={h[3]} it64={h[4]}" for h in r["history"])
        print(f"\n{name}: {rows}")
    assert abs(r64["stress"]) <= 1e-8
    assert abs(r32["stress"]) <= 1e-8
    assert abs(r64["history"][0][2]) > 1e-4  # L = 4.0 is far from stress-free
    # still the ordered (BCC) phase: the disordered phase, F = chiN fA (1 - fA) = 3.75, is
    # stress-free at every L
    assert r64["F"] < 3.75 - 1e-3 and r32["F"] < 3.75 - 1e-3
    assert abs(r32["L"] - r64["L"]) <= 1e-6
    assert abs(r32["F"] - r64["F"]) <= 1e-10 * abs(r64["F"])
    # the precision form's own stress (from its FP32 contour) against the FP64 adjoint, at the
    # start cell (large stress) and at the relaxed cell (stress ~ 0: absolute difference)
    w0 = (a, b)
    g64, g32 = _stress_at(G, 4.0, w0, "fp64"), _stress_at(G, 4.0, w0, "fp32")
    wr = (r64["wA"], r64["wB"])
    h64, h32 = _stress_at(G, r64["L"], wr, "fp64"), _stress_at(G, r64["L"], wr, "fp32")
    print(f"FP32 stress vs FP64 adjoint: L=4.0 {g32:+.9e} vs {g64:+.9e} (rel {abs(g32 - g64) / abs(g64):.2e}); "
          f"relaxed L={r64['L']:.9f}: {h32:+.3e} vs {h64:+.3e} (abs {abs(h32 - h64):.2e})")
    assert abs(g32 - g64) <= 1e-4 * abs(g64)
    assert abs(h32 - h64) <= 1e-6
    G.close()
