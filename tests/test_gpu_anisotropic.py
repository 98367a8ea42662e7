"""Orthorhombic PMMM (the reference's PMMM solver is cubic only, src/solver_Pmmm.h:101):
on a cell with Lx != Ly != Lz it must agree with P1 and 3M — which the reference does
support anisotropically — on the same mirror-symmetric fields: free energy, phi, and
the stress d ln Q / d L."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu

N = (32, 32, 48)
L = (4.2, 3.9, 5.6)


def _run(kind):
    wA, wB = fields.seed_fields(N, L, "BCC")
    if kind == "PMMM":
        G = solvers.CrysPSSolverPmmm(N, anisotropic=True)
    else:
        G = solvers.make_solver(kind, N)
    G.set_cell_para(L)
    assert np.allclose(G.get_cell_para()[:3], L)
    run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
    h = run.iterate(6)
    s = run.stress()
    f = run.get_fields()
    return h, s, fields.from_physical(kind, f["phiA"], N)


def test_anisotropic_pmmm_matches_p1_and_3m(gpu):
    hp, sp, php = _run("PMMM")
    for kind in ("P1", "3M"):
        h, s, ph = _run(kind)
        assert np.all(np.abs(hp["F"] - h["F"]) <= 1e-12 * np.abs(h["F"]))
        assert np.abs(php - ph).max() < 1e-12
        assert np.allclose(sp["dlnQ_dL"], s["dlnQ_dL"], rtol=1e-9, atol=1e-13)


def test_cubic_default_unchanged(gpu):
    G = solvers.CrysPSSolverPmmm(N)
    G.set_cell_para(L)
    assert np.allclose(G.get_cell_para()[:3], (L[0],) * 3)
