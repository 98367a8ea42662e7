"""Checkpoint and resume (crysscft_sample_b200.checkpoint): a run checkpointed after k
iterations and resumed in a new context continues exactly as the uninterrupted run."""
import numpy as np
import pytest

from crysscft_sample_b200 import checkpoint, fields, scft, solvers

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["PMMM", "3M"])
def test_resume_continues_the_run_exactly(gpu, tmp_path, kind):
    N, L = (32, 32, 32), 4.2
    wA, wB = fields.seed_fields(N, L, "BCC")
    a, b = fields.to_physical(kind, wA), fields.to_physical(kind, wB)

    def fresh():
        G = solvers.make_solver(kind, N)
        G.set_cell_para((L, L, L))
        run = scft.DiblockSCFT(G, 0.25, 0.01, 20.0, 0.1)
        run.set_fields(a, b)
        return run

    whole = fresh().iterate(8)["F"]
    first = fresh()
    h1 = first.iterate(5)["F"]
    first.save_checkpoint(tmp_path / "c.npz")
    meta, _ = checkpoint.read(tmp_path / "c.npz")
    assert meta["iterations"] == 5 and meta["kind"] == kind
    second = checkpoint.resume(tmp_path / "c.npz")
    assert second.iterations_done == 5
    h2 = second.iterate(3)["F"]
    assert np.array_equal(np.concatenate([h1, h2]), whole)
