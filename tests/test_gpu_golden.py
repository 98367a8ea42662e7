"""GPU results against the committed golden fixtures (outputs of the reference's own
solvers and driver loop, tests/golden/make_golden.py): one triplet per solver, and the
full 100-iteration run of the small BCC system for all three solvers (free energy
within 1e-10 relative every iteration, phi within 1e-12 max-abs)."""
import os

import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_triplets_match_golden(gpu):
    g = np.load(os.path.join(GOLDEN, "triplets.npz"))
    for kind, N in (("PMMM", (32, 32, 32)), ("3M", (32, 16, 48)), ("P1", (16, 24, 8))):
        k = f"{kind}_{N[0]}x{N[1]}x{N[2]}"
        G = solvers.make_solver(kind, N)
        G.set_cell_para(tuple(g[k + "_cell"]))
        G.set_contour_step(float(g[k + "_ds"]))
        io = G.get_iomat_for_diffusion()
        io[:] = g[k + "_in"]
        G.diffusion()
        assert np.abs(io - g[k + "_out"]).max() < 1e-13


@pytest.mark.parametrize("kind", ["PMMM", "3M", "P1"])
def test_100_iterations_match_golden(gpu, kind):
    g = np.load(os.path.join(GOLDEN, "scft_cfg0.npz"))
    N = (32, 32, 32)
    G = solvers.make_solver(kind, N)
    G.set_cell_para((4.2, 4.2, 4.2))
    run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    run.set_fields(fields.to_physical(kind, g["wA_full"]), fields.to_physical(kind, g["wB_full"]))
    h = run.iterate(100)
    F = g[kind + "_F"]
    assert np.all(np.abs(h["F"] - F) <= 1e-10 * np.abs(F))
    assert np.abs(h["maxinc"] - g[kind + "_maxinc"]).max() < 1e-10
    assert np.abs(h["Q"] - g[kind + "_Q"]).max() < 1e-11 * np.abs(g[kind + "_Q"]).max()
    assert np.abs(h["parts"] - g[kind + "_parts"]).max() < 1e-10
    if kind == "PMMM":
        f = run.get_fields()
        assert np.abs(f["phiA"] - g["PMMM_phiA"]).max() < 1e-12
        assert np.abs(f["phiB"] - g["PMMM_phiB"]).max() < 1e-12
        assert np.abs(f["wA"] - g["PMMM_wA_final"]).max() < 1e-11
