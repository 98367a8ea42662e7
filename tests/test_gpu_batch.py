"""Batching form: a batch of independent instances must reproduce, instance by
instance, the single-instance runs and the reference; every contour-kernel form gives
the same results; the autotuner restores the fields it advanced."""
import numpy as np
import pytest

from crysscft_sample_b200 import _lib, batch, fields, scft, solvers
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


def _mixed(n=10, seed=11):
    # every configured grid side (reduced 16, 24, 32, 48, 64) at least once
    cfg = batch.batch_config(n, seed=seed)
    for i, side in enumerate((16, 24, 32, 48, 64)):
        cfg[i]["N"] = (2 * side,) * 3
    return cfg


@pytest.mark.parametrize("teams", [None, {16: 1, 24: 1, 32: 1, 48: 1, 64: 1}, {16: 16, 24: 12, 32: 8, 48: 6, 64: 32}])
def test_one_launch_form_is_bit_identical_to_per_instance_kernels(gpu, teams):
    # form 4 runs each chain on a team of CTAs that own several planes / slabs each; every
    # unit does the per-instance kernel's arithmetic in the same order, so the results are
    # the same bits whatever the team sizes (the planner's, one CTA per chain, wide teams)
    inst = _mixed()
    B1 = batch.BatchSCFT("PMMM", inst)
    B1.configure(4, 1)
    B1.seed_fields()
    h1 = B1.iterate(3)
    B4 = batch.BatchSCFT("PMMM", inst)
    B4.configure(4, 4)
    if teams:
        B4.set_team_sizes(teams)
    B4.seed_fields()
    plan = B4.team_plan()
    assert plan["instances"] == len(inst) and plan["grid"] > 0
    assert B4.launches_per_iteration() < B1.launches_per_iteration()
    h4 = B4.iterate(3)
    assert np.array_equal(h4["F"], h1["F"])
    assert np.array_equal(h4["maxinc"], h1["maxinc"])
    for i in range(len(inst)):
        f1, f4 = B1.get_fields(i), B4.get_fields(i)
        for k in f1:
            assert np.array_equal(f4[k], f1[k]), f"instance {i} {k}"
    B1.close()
    B4.close()


def test_one_launch_form_timeout_is_reported_and_the_batch_survives(gpu):
    # a poll limit of 1: the first flag or tile-load wait of the batch kernel runs out; the
    # CTA sets the abort word, drains its own copies and leaves, the others stop waiting
    inst = _mixed(6, seed=3)
    ref_b = batch.BatchSCFT("PMMM", inst)
    ref_b.configure(4, 4)
    ref_b.seed_fields()
    want = ref_b.iterate(2)["F"]
    B = batch.BatchSCFT("PMMM", inst)
    B.configure(4, 4)
    B.seed_fields()
    B.iterate(1)
    B.set_wait_limit(1)
    with pytest.raises(_lib.ScftError) as e:
        B.iterate(1)
    assert e.value.status == 7  # SCFT_ERR_TIMEOUT
    B.set_wait_limit()
    B.seed_fields()
    got = B.iterate(2)["F"]
    assert np.array_equal(got, want)
    B.close()
    ref_b.close()


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
    tuned = B.autotune(2)
    B.configure(tuned["nstreams"], 4)  # the single persistent launch, whatever the autotuner chose
    assert B.team_plan()["instances"] == len(cfg)
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


def _run_forms(kind, inst, precision="fp64", n_iter=3):
    out = []
    for form in (1, 4):
        B = batch.BatchSCFT(kind, inst, precision=precision)
        B.configure(4, form)
        B.seed_fields()
        h = B.iterate(n_iter)
        plan = B.team_plan()
        fields_ = [B.get_fields(i) for i in range(len(inst))]
        B.close()
        out.append((h, plan, fields_))
    return out


def test_one_launch_form_with_instances_it_cannot_take(gpu):
    # physical 12^3 (not a multiple of 8) has no alternating kernel: that instance keeps its
    # own kernels on a worker stream, the others go to the one launch; the results match
    inst = _mixed(6, seed=13)
    inst[1]["N"] = (24, 24, 24)
    (h1, _, f1), (h4, plan, f4) = _run_forms("PMMM", inst)
    assert plan["instances"] == len(inst) - 1
    assert np.array_equal(h4["F"], h1["F"])
    for a, b in zip(f1, f4):
        assert all(np.array_equal(a[k], b[k]) for k in a)


def test_one_launch_form_p1_batch(gpu):
    # P1 (one even/odd level on every axis) through the same batch kernel
    inst = batch.batch_config(4, seed=21, sizes=(8, 16, 24, 32))
    (h1, _, _), (h4, plan, _) = _run_forms("P1", inst)
    assert plan["instances"] == len(inst)
    assert np.array_equal(h4["F"], h1["F"])


def test_one_launch_form_leaves_fp32_instances_to_their_kernels(gpu):
    # the batch kernel is FP64; an FP32 batch in form 4 plans no team and runs as form 0
    inst = _mixed(5, seed=17)
    (h1, _, _), (h4, plan, _) = _run_forms("PMMM", inst, precision="fp32")
    assert plan["instances"] == 0 and plan["grid"] == 0
    assert np.array_equal(h4["F"], h1["F"])
