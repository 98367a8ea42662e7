"""GPU SCFT iteration parity against the reference's own driver loop (oracle/_ref):
per-iteration free energy within 1e-10 relative and phi within 1e-12 max-abs."""
import numpy as np
import pytest

from oracle import ref
from crysscft_sample_b200 import fields, scft, solvers

pytestmark = pytest.mark.gpu

F_RTOL = 1e-10
PHI_ATOL = 1e-12

# the small BCC system: 32^3 full grid, L=4.2, fA=0.25, chiN=20, ds=0.01, lambda=0.1
CFG0 = dict(N=(32, 32, 32), L=4.2, fA=0.25, xN=20.0, ds=0.01, acc=0.1)


def _run_pair(kind, cfg, nstep, precision="fp64"):
    N, L = cfg["N"], cfg["L"]
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    R = ref.RefSolver(kind, N)
    want = R.scft_run(cfg["fA"], cfg["ds"], cfg["xN"], (L, L, L), cfg["acc"], nstep, a, b)
    G = solvers.make_solver(kind, N, precision=precision)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, cfg["fA"], cfg["ds"], cfg["xN"], cfg["acc"])
    run.set_fields(a, b)
    got = run.iterate(nstep)
    got.update(run.get_fields())
    return want, got


@pytest.mark.parametrize("kind", ["PMMM", "3M", "P1"])
def test_iterations_match_reference(gpu, kind):
    want, got = _run_pair(kind, CFG0, 20)
    _compare(want, got)


# grids that exercise every launch form: persistent kernel with even/odd axes (64^3 PMMM,
# 64^3 P1), full-matrix axes (3M), mixed axes (48 = not a multiple of 16), and the
# per-axis fallback kernels (36 -> 18 is not a multiple of 8; 128 is above the
# persistent kernel's plane limit)
SIZES = [
    ("PMMM", (128, 128, 128), 2),
    ("3M", (128, 128, 128), 2),
    ("P1", (64, 64, 64), 2),
    ("PMMM", (96, 64, 32), 3),
    ("3M", (36, 32, 48), 3),
    ("P1", (128, 32, 16), 2),
    # alternating kernel with 5, 6 and 7 column panels per tile (40^3 one level, 48^3 even/odd,
    # 56^3 one level)
    ("P1", (40, 40, 40), 2),
    ("PMMM", (96, 96, 96), 2),
    ("P1", (56, 56, 56), 2),
]


@pytest.mark.parametrize("kind,N,nstep", SIZES)
def test_iterations_match_reference_sizes(gpu, kind, N, nstep):
    cfg = dict(CFG0, N=N, ds=0.005)
    want, got = _run_pair(kind, cfg, nstep)
    _compare(want, got)


# the FP64 tensor-core axis passes of large cubic grids (128^3 physical: PMMM and 3M on a
# 256^3 full grid, P1 on 128^3; 96^3 physical: PMMM on 192^3), on a shorter contour
LARGE = [
    ("PMMM", (256, 256, 256)),
    ("3M", (256, 256, 256)),
    ("P1", (128, 128, 128)),
    ("PMMM", (192, 192, 192)),
]


@pytest.mark.parametrize("kind,N", LARGE)
def test_iterations_match_reference_large(gpu, kind, N):
    cfg = dict(CFG0, N=N, ds=0.02)
    want, got = _run_pair(kind, cfg, 2)
    _compare(want, got)


def _compare(want, got):
    assert np.all(np.abs(got["F"] - want["F"]) <= F_RTOL * np.abs(want["F"]))
    assert np.abs(got["maxinc"] - want["maxinc"]).max() < 1e-11
    assert np.abs(got["Q"] - want["Q"]).max() < 1e-12 * np.abs(want["Q"]).max()
    assert np.abs(got["parts"] - want["parts"]).max() < 1e-11
    assert np.abs(got["phiA"] - want["phiA"]).max() < PHI_ATOL
    assert np.abs(got["phiB"] - want["phiB"]).max() < PHI_ATOL
    assert np.abs(got["wA"] - want["wA"]).max() < 1e-11


def test_host_buffer_iteration_matches_device_iteration(gpu):
    # the end-to-end form (fields in from host arrays, phi and fields back every call)
    N, L = CFG0["N"], CFG0["L"]
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical("PMMM", wA).ravel(), fields.to_physical("PMMM", wB).ravel()

    def ctx():
        G = solvers.make_solver("PMMM", N)
        G.set_cell_para((L, L, L))
        return scft.DiblockSCFT(G, CFG0["fA"], CFG0["ds"], CFG0["xN"], CFG0["acc"])

    dev = ctx()
    dev.set_fields(a, b)
    want = dev.iterate(3)
    want.update(dev.get_fields())
    host = ctx()
    ha, hb = a.copy(), b.copy()
    pa, pb = np.empty_like(ha), np.empty_like(hb)
    F = []
    for _ in range(3):
        F.append(host.iterate_host(ha, hb, 1, pa, pb)["F"][0])
    assert np.array_equal(np.array(F), want["F"])
    assert np.array_equal(pa, want["phiA"]) and np.array_equal(pb, want["phiB"])
    assert np.array_equal(ha, want["wA"]) and np.array_equal(hb, want["wB"])
    # several iterations in one call: every history row comes back
    multi = ctx()
    ma, mb = a.copy(), b.copy()
    got = multi.iterate_host(ma, mb, 3)
    for key in ("F", "Q", "maxinc", "parts"):
        assert np.array_equal(got[key], want[key]), key
    assert np.array_equal(got["phiA"], want["phiA"]) and np.array_equal(ma, want["wA"])
