"""The FFT ("butterfly") form of the FP64 axis passes against the reference's own triplets
and against the dense form.

Every axis operator is a real circulant with an even spectrum on an extension of the line
(P1: the line; PMMM: the mirror extension, DCT-II/III; 3m: the interleaved mirror extension
of the even sub-lattice), applied with complex FFTs of two lines at once.  CRYSSCFT_AXIS_FORM
selects the form (fft / dense).
"""
import os

import numpy as np
import pytest

from crysscft_sample_b200 import scft, solvers
from oracle import ref

pytestmark = pytest.mark.gpu

CASES = [
    ("PMMM", (64, 64, 64)), ("PMMM", (128, 128, 128)), ("PMMM", (256, 256, 256)),
    ("3M", (64, 64, 64)), ("3M", (256, 256, 256)),
    ("P1", (64, 64, 64)), ("P1", (128, 128, 128)), ("P1", (256, 256, 256)),
    ("PMMM", (128, 64, 256)),  # axes with transform lengths 128, 64 and 256 in one triplet
]


class _Form:
    """CRYSSCFT_AXIS_FORM set for the duration of a block."""

    def __init__(self, form):
        self.form = form

    def __enter__(self):
        self.old = os.environ.get("CRYSSCFT_AXIS_FORM")
        os.environ["CRYSSCFT_AXIS_FORM"] = self.form

    def __exit__(self, *exc):
        if self.old is None:
            del os.environ["CRYSSCFT_AXIS_FORM"]
        else:
            os.environ["CRYSSCFT_AXIS_FORM"] = self.old


def _cell(kind, L):
    return (L[0],) * 3 if kind == "PMMM" else L


def _triplet(kind, N, q, form, L=(4.2, 3.9, 5.1), ds=0.005):
    with _Form(form):
        G = solvers.make_solver(kind, N)
        G.set_cell_para(_cell(kind, L))
        G.set_contour_step(ds)
        io = G.get_iomat_for_diffusion()
        io[:] = q
        G.diffusion()
        out = io.copy()
        G.close()
    return out


@pytest.mark.parametrize("kind,N", CASES)
def test_fft_triplet_matches_reference(gpu, kind, N):
    rng = np.random.default_rng(3)
    L = (4.2, 3.9, 5.1)
    R = ref.RefSolver(kind, N)
    R.set_cell_para(_cell(kind, L))
    R.set_contour_step(0.005)
    q = rng.random(R.space_size_phy) + 0.5
    want = R.diffusion(q)
    R.close()
    got = _triplet(kind, N, q, "fft")
    assert np.abs(got - want).max() < 1e-13
    dense = _triplet(kind, N, q, "dense")
    assert np.abs(got - dense).max() < 1e-13
    assert not np.array_equal(got, dense)  # two different kernels ran (they round differently)


def test_fft_propagation_matches_reference(gpu):
    # a 20-step chain with the Boltzmann factors fused into the first and last pass
    kind, N, L, ds = "PMMM", (256, 256, 256), (4.2,) * 3, 0.005
    rng = np.random.default_rng(4)
    R = ref.RefSolver(kind, N)
    R.set_cell_para(L)
    R.set_contour_step(ds)
    M = R.space_size_phy
    init = np.ones(M)
    wds = np.exp(-0.5 * ds * (1.0 + 0.3 * rng.standard_normal(M)))
    want = R.solve_diffusion_equation(init, wds, 20, 1)
    R.close()
    with _Form("fft"):
        G = solvers.make_solver(kind, N)
        G.set_cell_para(L)
        G.set_contour_step(ds)
        got = scft.solve_diffusion_equation(np.zeros(21 * M), init, wds, G, 20, 1)
        G.close()
    assert np.abs(got.reshape(21, M) - want).max() < 1e-12


@pytest.mark.parametrize("kind,n", [("PMMM", 256), ("P1", 256)])
def test_fft_iterations_match_dense(gpu, kind, n):
    # two SCFT iterations at 256^3 (Ns = 200) through the FFT passes against the dense passes
    from crysscft_sample_b200 import fields

    N, L = (n, n, n), 4.2
    wA, wB = fields.seed_fields(N, L, "BCC")
    out = {}
    for form in ("fft", "dense"):
        with _Form(form):
            G = solvers.make_solver(kind, N)
            G.set_cell_para((L, L, L))
            run = scft.DiblockSCFT(G, 0.25, 0.005, 20.0, 0.1)
            run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
            out[form] = run.iterate(2)
            out[form].update(run.get_fields())
            run.close()
            G.close()
    rel = np.abs(out["fft"]["F"] - out["dense"]["F"]) / np.abs(out["dense"]["F"])
    assert rel.max() < 1e-12
    assert not np.array_equal(out["fft"]["phiA"], out["dense"]["phiA"])  # both forms really ran
    assert np.abs(out["fft"]["phiA"] - out["dense"]["phiA"]).max() < 1e-12


@pytest.mark.parametrize("kind,n", [("PMMM", 256), ("P1", 128)])
def test_fp32_fft_iterations_track_fp64(gpu, kind, n):
    # the precision form's triplets by FP32 FFT (round-to-nearest CUDA-core arithmetic): its
    # iterations track FP64 as closely as the 3xTF32 dense passes do
    from crysscft_sample_b200 import fields

    N, L = (n, n, n), 4.2
    wA, wB = fields.seed_fields(N, L, "BCC")
    F = {}
    for form, prec in (("dense", "fp64"), ("fft", "fp32"), ("dense", "fp32")):
        with _Form(form):
            G = solvers.make_solver(kind, N)
            G.set_cell_para((L, L, L))
            run = scft.DiblockSCFT(G, 0.25, 0.005, 20.0, 0.1)
            run.set_fields(fields.to_physical(kind, wA), fields.to_physical(kind, wB))
            run.set_precision(prec)
            F[(form, prec)] = run.iterate(3)["F"]
            run.close()
            G.close()
    ref64 = F[("dense", "fp64")]
    rel_fft = np.abs(F[("fft", "fp32")] - ref64) / np.abs(ref64)
    rel_tf32 = np.abs(F[("dense", "fp32")] - ref64) / np.abs(ref64)
    print(f"\n{kind} {n}^3 FP32 |dF/F| vs FP64: FFT {rel_fft.max():.3e}, 3xTF32 dense {rel_tf32.max():.3e}")
    assert 1e-12 < rel_fft.max() < 3e-5
    assert not np.array_equal(F[("fft", "fp32")], F[("dense", "fp32")])
