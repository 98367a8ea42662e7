"""Precision form: FP32 triplets (3xTF32 tensor-core split products) with FP64 Q, phi,
free energy and mixing, finished by FP64 polish iterations.  Errors are measured
against the FP64 reference (oracle/_ref) on the same seeded fields."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields, scft, solvers
from oracle import ref

pytestmark = pytest.mark.gpu

FP32_REL = 3e-5      # FP32 triplets: per-iteration |dF/F| (~8e-6 measured: 600 chained FP32 axis products)
POLISHED_REL = 1e-8  # after the FP64 polish (the precision form's target)


def _pair(kind, N, nstep, npolish, L=4.2, fA=0.25, xN=20.0, ds=0.01, acc=0.1):
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)
    want = ref.RefSolver(kind, N).scft_run(fA, ds, xN, (L, L, L), acc, nstep, a, b)
    G = solvers.make_solver(kind, N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, fA, ds, xN, acc)
    run.set_fields(a, b)
    got = run.iterate_polished(nstep, npolish)
    got.update(run.get_fields())
    return want, got


@pytest.mark.parametrize("kind,N", [("PMMM", (32, 32, 32)), ("3M", (32, 32, 32)), ("P1", (32, 32, 32)),
                                    ("PMMM", (64, 64, 64)), ("PMMM", (128, 128, 128))])
def test_fp32_triplets_track_fp64(gpu, kind, N):
    # PMMM 128^3 (64^3 physical) is the FP32 contour kernel of the 128^3 BCC benchmark
    want, got = _pair(kind, N, 6, 1)
    rel = np.abs(got["F"] - want["F"]) / np.abs(want["F"])
    assert rel[:-1].max() < FP32_REL          # FP32 iterations
    assert rel[-1] < rel[:-1].max() / 10      # one FP64 iteration removes most of the FP32 error
    assert rel[:-1].max() > 1e-12             # the FP32 path really ran in FP32


@pytest.mark.parametrize("kind,N", [("PMMM", (256, 256, 256)), ("P1", (128, 128, 128))])
def test_fp32_large_grid_axis_passes_track_fp64(gpu, kind, N):
    # 128^3 physical: the FP32 triplets run as 3xTF32 tensor-core axis passes
    want, got = _pair(kind, N, 3, 1, ds=0.02)
    rel = np.abs(got["F"] - want["F"]) / np.abs(want["F"])
    assert rel[:-1].max() < FP32_REL
    assert rel[-1] < rel[:-1].max() / 10
    assert rel[:-1].max() > 1e-12


@pytest.mark.parametrize("kind", ["PMMM", "P1"])
def test_fp32_plus_polish_reaches_target(gpu, kind):
    want, got = _pair(kind, (32, 32, 32), 40, 2)
    assert abs(got["F"][-1] - want["F"][-1]) <= POLISHED_REL * abs(want["F"][-1])
    assert np.abs(got["phiA"] - want["phiA"]).max() < 1e-5  # trajectory difference left by FP32


def test_precision_switch_round_trip(gpu):
    G = solvers.CrysPSSolverPmmm((32, 32, 32))
    G.set_cell_para((4.2, 4.2, 4.2))
    run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    wA, wB = fields.seed_fields((32, 32, 32), 4.2)
    run.set_fields(fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
    assert run.get_precision() == "fp64"
    run.set_precision("fp32")
    assert run.get_precision() == "fp32"
    h = run.iterate(2)
    assert np.all(np.isfinite(h["F"]))
    run.set_precision("fp64")
    assert np.all(np.isfinite(run.iterate(1)["F"]))


def test_switching_precision_back_and_forth_replays_saved_graphs(gpu):
    # each precision keeps its captured iteration graph; buffers those graphs use must
    # survive the other precision's setup (FP32 -> FP64 -> FP32 replays the FP32 graph)
    def sequence():
        N, L = (64, 64, 64), 4.2
        wA, wB = fields.seed_fields(N, L, "BCC")
        G = solvers.make_solver("PMMM", N)
        G.set_cell_para((L, L, L))
        run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
        run.set_fields(fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
        out = []
        for precision, n in (("fp32", 2), ("fp64", 1), ("fp32", 2), ("fp64", 1)):
            run.set_precision(precision)
            out.append(run.iterate(n)["F"])
        return np.concatenate(out)

    a, b = sequence(), sequence()
    assert np.all(np.isfinite(a))
    assert np.array_equal(a, b)
