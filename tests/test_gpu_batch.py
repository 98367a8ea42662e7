"""Batching form: a batch of independent instances must reproduce, instance by
instance, the single-instance runs and the reference; every contour-kernel form gives
the same results; the autotuner restores the fields it advanced."""
import numpy as np
import pytest

from crysscft_sample_b200 import batch, fields, scft, solvers
from oracle import ref

pytestmark = pytest.mark.gpu


def _instances():
    cfg = batch.batch_config(6, seed=7, sizes=(8, 16, 24, 32))
    cfg[0]["N"] = (32, 32, 32)  # make sure a 16^3 physical grid is present
    return cfg


def _single(inst, n_iter, ds=0.01):
    G = solvers.make_solver("PMMM", inst["N"])
    G.set_cell_para((inst["L"],) * 3)
    run = scft.DiblockSCFT(G, inst["fA"], ds, inst["xN"], 0.1)
    wA, wB = fields.seed_fields(inst["N"], inst["L"], inst["phase"], seed=inst["seed"])
    run.set_fields(fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
    h = run.iterate(n_iter)
    h.update(run.get_fields())
    return h


def test_batch_matches_single_instance_runs(gpu):
    inst = _instances()
    B = batch.BatchSCFT("PMMM", inst)
    B.seed_fields()
    hb = B.iterate(4)
    for i, it in enumerate(inst):
        hs = _single(it, 4)
        assert np.allclose(hb["F"][:, i], hs["F"], rtol=1e-12, atol=0)
        assert np.abs(B.get_fields(i)["phiA"] - hs["phiA"]).max() < 1e-13
    # caller-provided output arrays receive the same fields
    for i in range(len(inst)):
        out = [np.full(B.M[i], np.nan) for _ in range(4)]
        got = B.get_fields(i, out=out)
        want = B.get_fields(i)
        assert all(got[k] is out[j] for j, k in enumerate(("phiA", "phiB", "wA", "wB")))
        assert all(np.array_equal(got[k], want[k]) for k in want)
    with pytest.raises(ValueError):
        B.get_fields(0, out=[np.empty(3)] * 4)


def test_batch_instance_matches_reference(gpu):
    inst = _instances()
    B = batch.BatchSCFT("PMMM", inst)
    B.seed_fields()
    hb = B.iterate(3)
    it = inst[0]
    wA, wB = fields.seed_fields(it["N"], it["L"], it["phase"], seed=it["seed"])
    want = ref.RefSolver("PMMM", it["N"]).scft_run(it["fA"], 0.01, it["xN"], (it["L"],) * 3, 0.1, 3,
                                                   fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
    assert np.all(np.abs(hb["F"][:, 0] - want["F"]) <= 1e-10 * np.abs(want["F"]))


@pytest.mark.parametrize("form", [1, 2, 3])
def test_every_kernel_form_agrees(gpu, form):
    inst = _instances()
    B0 = batch.BatchSCFT("PMMM", inst)
    B0.seed_fields()
    h0 = B0.iterate(3)
    B = batch.BatchSCFT("PMMM", inst)
    B.configure(3, form)
    B.seed_fields()
    h = B.iterate(3)
    assert np.allclose(h["F"], h0["F"], rtol=1e-11, atol=0)


def test_autotune_restores_fields(gpu):
    inst = _instances()
    B = batch.BatchSCFT("PMMM", inst)
    B.seed_fields()
    best = B.autotune(2)
    assert best["nstreams"] >= 1 and best["ms_per_iteration"] > 0
    h = B.iterate(2)
    B2 = batch.BatchSCFT("PMMM", inst)
    B2.seed_fields()
    h2 = B2.iterate(2)
    assert np.allclose(h["F"], h2["F"], rtol=1e-11, atol=0)


def test_batching_configuration_200_iterations(gpu):
    # the configured batch: 64 seeded PMMM instances, reduced grids from {16, 24, 32, 48, 64}^3,
    # chiN ~ U[14, 30], fA ~ U[0.2, 0.35], L ~ U[3.8, 5.5], BCC or FCC, 200 iterations each
    # (ds = 0.01), one graph launch per batch iteration after the autotuner's choice; every
    # instance against its single-instance run, the three smallest against the reference
    cfg = batch.batch_config(64)
    B = batch.BatchSCFT("PMMM", cfg, ds=0.01)
    B.seed_fields()
    B.autotune(2)
    hb = B.iterate(200)
    assert np.all(np.isfinite(hb["F"]))
    for i, it in enumerate(cfg):
        hs = _single(it, 200)
        rel = np.abs(hb["F"][:, i] - hs["F"]) / np.abs(hs["F"])
        assert rel.max() <= 1e-10, f"instance {i} ({it['N']}): max |dF/F| {rel.max():.3e}"
    B.close()
    small = sorted(range(len(cfg)), key=lambda i: (cfg[i]["N"][0], i))[:3]
    for i in small:
        it = cfg[i]
        wA, wB = fields.seed_fields(it["N"], it["L"], it["phase"], seed=it["seed"])
        want = ref.RefSolver("PMMM", it["N"]).scft_run(it["fA"], 0.01, it["xN"], (it["L"],) * 3, 0.1, 200,
                                                       fields.to_physical("PMMM", wA),
                                                       fields.to_physical("PMMM", wB))
        rel = np.abs(hb["F"][:, i] - want["F"]) / np.abs(want["F"])
        assert rel.max() <= 1e-10, f"instance {i} ({it['N']}) vs reference: max |dF/F| {rel.max():.3e}"
