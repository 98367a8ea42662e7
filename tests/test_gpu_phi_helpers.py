"""The density integral inside the contour launch: the FP64 alternating kernel runs blocks
on the SMs its units leave free, which sum w_s q(s) q+(s) over the interior contour slots
as the two chains store them (src/crysSCFT_sample.cpp:348-360); a short kernel adds the
end slots and the 1/(Ns Q) factors.  Checks: the same iterations as the separate phi pass
(CRYSSCFT_PHI_HELPERS=0) to the rounding level, and against the reference's own driver
loop (oracle/_ref) on a small grid, where the helpers outnumber the units."""
import numpy as np
import pytest

from oracle import ref
from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu


def _iterate(kind, N, L, nstep, helpers, monkeypatch, ds=0.005):
    if helpers is None:
        monkeypatch.delenv("CRYSSCFT_PHI_HELPERS", raising=False)
    else:
        monkeypatch.setenv("CRYSSCFT_PHI_HELPERS", helpers)
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    G = solvers.make_solver(kind, N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, 0.25, ds, 20.0, 0.1)
    run.set_fields(a, b)
    h = run.iterate(nstep)
    h.update(run.get_fields())
    run.close()
    G.close()
    return h, a, b


@pytest.mark.parametrize("kind", ["PMMM", "P1"])
def test_helpers_match_the_separate_pass(gpu, kind, monkeypatch):
    N = (128, 128, 128) if kind == "PMMM" else (64, 64, 64)  # 64^3 physical: the bench grid
    on, _, _ = _iterate(kind, N, 4.2, 4, None, monkeypatch)
    off, _, _ = _iterate(kind, N, 4.2, 4, "0", monkeypatch)
    rel = np.abs(on["F"] - off["F"]) / np.abs(off["F"])
    dphi = max(np.abs(on["phiA"] - off["phiA"]).max(), np.abs(on["phiB"] - off["phiB"]).max())
    print(f"\n{kind} {N}: helpers vs separate pass |dF/F| {rel.max():.2e}, max |dphi| {dphi:.2e}")
    assert rel.max() <= 1e-13
    assert dphi <= 1e-14
    assert not np.array_equal(on["phiA"], off["phiA"])  # the two forms really ran (they round differently)


def test_helpers_match_reference_small_grid(gpu, monkeypatch):
    # 64^3 PMMM (32^3 physical): 64 units, the other SMs' blocks sum ~400 points each
    kind, N, L, n = "PMMM", (64, 64, 64), 4.2, 6
    got, a, b = _iterate(kind, N, L, n, "1", monkeypatch, ds=0.01)
    want = ref.RefSolver(kind, N).scft_run(0.25, 0.01, 20.0, (L, L, L), 0.1, n, a, b)
    assert np.allclose(got["F"], want["F"], rtol=1e-10, atol=0)
    assert np.abs(got["phiA"] - want["phiA"]).max() <= 1e-12
    assert np.abs(got["phiB"] - want["phiB"]).max() <= 1e-12
    off, _, _ = _iterate(kind, N, L, n, "0", monkeypatch, ds=0.01)
    assert not np.array_equal(got["phiA"], off["phiA"])
