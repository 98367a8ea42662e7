"""phi summed inside the whole-contour kernel against the separate pass over the stored
contour (integrate_phi, src/crysSCFT_sample.cpp:348-360).

The alternating kernel adds q(s) q+(s) for the slots of the contour's second half as the
second chain reaches them; a short kernel adds slots 0, NsA, U/2 and U with their
trapezoid weights.  Both forms must give the same free energy and phi up to the order of
the sums.  The cases put the block boundary NsA below, at and above the midpoint U/2, run
the bench system (64^3 physical, Ns = 200), a one-level P1 grid, an odd step count (the
fused form is off there and the separate pass runs) and the FP32 contour kernel of the
precision form (FP32 tiles, FP64 products and sums).  The reference parity of the
default (fused) form is the iteration tests' job.
"""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu

F_RTOL = 1e-13
PHI_ATOL = 1e-13

CASES = [
    # kind, full grid, fA, ds, iterations, precision of the triplets: NsA / NsB
    ("PMMM", (128, 128, 128), 0.25, 0.005, 3, "fp64"),  # 50 / 150, the bench system
    ("PMMM", (32, 32, 32), 0.5, 0.01, 4, "fp64"),  # 50 / 50: NsA = U / 2
    ("PMMM", (32, 32, 32), 0.7, 0.01, 4, "fp64"),  # 70 / 30: NsA above the midpoint
    ("P1", (32, 32, 32), 0.25, 0.01, 4, "fp64"),  # one-level operators
    ("PMMM", (64, 64, 64), 0.3, 0.0102, 4, "fp64"),  # 29 / 68: U odd, separate pass either way
    # FP32 contour kernel: FP32 tiles, products and sums in FP64
    ("PMMM", (128, 128, 128), 0.25, 0.005, 3, "fp32"),
    ("PMMM", (64, 64, 64), 0.5, 0.01, 3, "fp32"),
    ("PMMM", (64, 64, 64), 0.7, 0.01, 3, "fp32"),
]


def _run(kind, N, fA, ds, nit, fused, precision="fp64"):
    L = 4.2
    wA, wB = fields.seed_fields(N, L, "BCC")
    G = solvers.make_solver(kind, N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, fA, ds, 20.0, 0.1)
    run.set_precision(precision)
    run.set_phi_form(fused)
    run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
    h = run.iterate(nit)
    h.update(run.get_fields())
    run.close()
    G.close()
    return h


@pytest.mark.parametrize("kind,N,fA,ds,nit,precision", CASES)
def test_fused_phi_matches_separate_pass(gpu, kind, N, fA, ds, nit, precision):
    a = _run(kind, N, fA, ds, nit, True, precision)
    b = _run(kind, N, fA, ds, nit, False, precision)
    rel = np.abs(a["F"] - b["F"]) / np.abs(b["F"])
    assert rel.max() <= F_RTOL, f"F rel diff {rel.max():.2e}"
    for k in ("phiA", "phiB"):
        d = np.abs(a[k] - b[k]).max()
        assert d <= PHI_ATOL, f"{k} max |fused - separate| = {d:.2e}"
    assert np.isfinite(a["phiA"]).all() and a["phiA"].max() > 0


def test_phi_form_switch_between_runs(gpu):
    # one run object, the form switched between iterate() calls: the captured iteration
    # graph is rebuilt and the fields carry on
    N, L = (32, 32, 32), 4.2
    wA, wB = fields.seed_fields(N, L, "BCC")
    a0, b0 = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)
    G = solvers.make_solver("PMMM", N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    run.set_fields(a0, b0)
    h1 = run.iterate(2)
    run.set_phi_form(False)
    h2 = run.iterate(2)
    run.set_phi_form(True)
    h3 = run.iterate(2)
    ref = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    ref.set_phi_form(False)
    ref.set_fields(a0, b0)
    hr = ref.iterate(6)
    got = np.concatenate([h1["F"], h2["F"], h3["F"]])
    assert (np.abs(got - hr["F"]) / np.abs(hr["F"])).max() <= F_RTOL
    run.close()
    ref.close()
    G.close()
