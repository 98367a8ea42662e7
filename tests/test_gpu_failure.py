"""Failure detection on the GPU without a GPU fault.  A bounded device wait that runs
out (a poll limit of 1 on the contour kernel's flag, barrier and tile-load waits) ends
the launch with SCFT_ERR_TIMEOUT and leaves the context usable; non-finite fields are
reported as SCFT_ERR_NUMERIC; a device allocation that cannot fit is SCFT_ERR_ALLOC.
(The reference prints "ERROR" and exits instead.)"""
import numpy as np
import pytest

from crysscft_sample_b200 import _lib, fields, scft, solvers
from crysscft_sample_b200._lib import ScftError

pytestmark = pytest.mark.gpu

N, L = (64, 64, 64), 4.2


def _fresh():
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)
    G = solvers.make_solver("PMMM", N)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
    run.set_fields(a, b)
    return run, a, b


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_a_wait_that_runs_out_is_a_timeout_and_the_context_survives(gpu, precision):
    ref, a, b = _fresh()
    ref.set_precision(precision)
    want = ref.iterate(2)["F"]
    run, _, _ = _fresh()
    run.set_precision(precision)
    run.iterate(1)  # graphs captured with the default limit first
    run.set_wait_limit(1)
    with pytest.raises(ScftError) as e:
        run.iterate(1)
    assert e.value.status == 7  # SCFT_ERR_TIMEOUT
    run.set_wait_limit()
    run.set_fields(a, b)  # the failed iteration's fields are not to be trusted
    got = run.iterate(2)["F"]
    assert np.array_equal(got, want)


def test_cluster_kernel_timeout_drains_and_the_context_survives(gpu, monkeypatch):
    # the FP32 cluster kernel (tcgen05 MMAs, bulk copies, cluster barriers): a wait that runs
    # out makes every CTA skip its work but keep the cluster barriers, drain its own MMAs and
    # copies, free its tensor memory and return; the call reports SCFT_ERR_TIMEOUT and the
    # context then reproduces a fresh run
    monkeypatch.setenv("CRYSSCFT_FP32_CLUSTER", "1")
    n = (128, 128, 128)  # 64^3 physical: the grid the cluster kernel runs
    wA, wB = fields.seed_fields(n, L, "BCC")
    a, b = fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB)

    def fresh():
        G = solvers.make_solver("PMMM", n)
        G.set_cell_para((L, L, L))
        r = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
        r.set_fields(a, b)
        r.set_precision("fp32")
        return r

    want = fresh().iterate(2)["F"]
    monkeypatch.setenv("CRYSSCFT_FP32_CLUSTER", "0")
    assert not np.array_equal(fresh().iterate(2)["F"], want)  # the cluster kernel really ran
    monkeypatch.setenv("CRYSSCFT_FP32_CLUSTER", "1")
    run = fresh()
    run.iterate(1)
    run.set_wait_limit(1)
    with pytest.raises(ScftError) as e:
        run.iterate(1)
    assert e.value.status == 7  # SCFT_ERR_TIMEOUT
    run.set_wait_limit()
    run.set_fields(a, b)
    assert np.array_equal(run.iterate(2)["F"], want)


def test_non_finite_fields_are_a_numeric_error(gpu):
    run, a, b = _fresh()
    bad = a.copy()
    bad.ravel()[123] = np.nan
    run.set_fields(bad, b)
    with pytest.raises(ScftError) as e:
        run.iterate(1)
    assert e.value.status == 6  # SCFT_ERR_NUMERIC
    run.set_fields(a, b)
    assert np.all(np.isfinite(run.iterate(1)["F"]))


def test_a_contour_store_that_cannot_fit_is_an_allocation_error(gpu):
    # 256^3 physical grid, ds = 0.0005: 2001 slices x 134 MB per chain, more than the device
    G = solvers.make_solver("PMMM", (512, 512, 512))
    G.set_cell_para((L, L, L))
    with pytest.raises(ScftError) as e:
        scft.DiblockSCFT(G, 0.25, 0.0005, 20.0, 0.1)
    assert e.value.status == 4  # SCFT_ERR_ALLOC
    G.close()


def test_solver_and_context_may_be_destroyed_in_either_order(gpu):
    run, a, b = _fresh()
    G = run.solver
    G.close()              # deferred: the context still uses the solver
    assert np.all(np.isfinite(run.iterate(1)["F"]))
    run.close()            # frees the context, then the solver
    run2, _, _ = _fresh()
    run2.close()
    run2.solver.close()
