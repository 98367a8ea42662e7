"""Run the configured AB-diblock system for a few iterations (or triplets) and print F.

    python -m crysscft_sample_b200.run [--solver PMMM|3M|P1] [--grid 128] [--phase BCC|FCC]
        [--precision fp64|fp32] [--iterations 3] [--triplets 0] [--ds 0.005]
        [--batch K [--batch-form 4]]

The systems are the seeded ones of the benchmark and the tests (BCC: L = 4.2, fA = 0.25,
chiN = 20; FCC: L = 5.0, fA = 0.22, chiN = 25; simple mixing lambda = 0.1).  --triplets K runs K
triplets through scft_solver_diffusion_device instead of iterations and prints their
CUDA-event time.  --batch K runs the seeded batching workload with K instances (reduced
grids from {16, 24, 32, 48, 64}^3, ds = 0.01) in contour form --batch-form (4: all contours
in one persistent launch) and prints each instance's last F.  The first iteration
(triplet) runs before the reported ones, so a profiler can skip the set-up launches.
CRYSSCFT_AXIS_FORM=fft|dense and CRYSSCFT_FP32_CLUSTER=1 select kernel forms.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

SYSTEMS = {"BCC": dict(L=4.2, fA=0.25, xN=20.0), "FCC": dict(L=5.0, fA=0.22, xN=25.0)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--solver", choices=["PMMM", "3M", "P1"], default="PMMM")
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--phase", choices=list(SYSTEMS), default="BCC")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--iterations", type=int, default=3)
    ap.add_argument("--triplets", type=int, default=0)
    ap.add_argument("--ds", type=float, default=0.005)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--batch-form", type=int, default=4)
    a = ap.parse_args(argv)

    import torch

    from . import batch, fields, scft, solvers

    if a.batch:
        B = batch.BatchSCFT("PMMM", batch.batch_config(a.batch), ds=0.01)
        B.seed_fields()
        B.configure(4, a.batch_form)
        print("plan:", B.team_plan() if a.batch_form == 4 else "one contour kernel per instance")
        B.iterate(1)
        h = B.iterate(a.iterations)
        for i, F in enumerate(h["F"][-1]):
            print(f"instance {i} {B.instances[i]['N']}: F = {F:.12f}")
        B.close()
        return 0

    sysp = SYSTEMS[a.phase]
    N = (a.grid,) * 3
    G = solvers.make_solver(a.solver, N)
    G.set_cell_para((sysp["L"],) * 3)
    if a.triplets:
        G.set_contour_step(a.ds)
        M = G.get_space_size_phy()
        stream = torch.cuda.Stream()  # the solver's work and the timing events on one stream
        G.set_stream(stream)
        q = torch.tensor(np.random.default_rng(1).random(M) + 0.5, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        G.diffusion_device(q, stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.triplets):
            G.diffusion_device(q, stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / a.triplets
        print(f"{a.triplets} triplets on {G.get_grid_size_phy()} physical: {ms * 1e3:.1f} us per triplet "
              f"({1e3 / ms:.0f} triplets/s), mean {q.mean().item():.12f}")
        G.close()
        return 0
    wA, wB = fields.seed_fields(N, sysp["L"], a.phase)
    run = scft.DiblockSCFT(G, sysp["fA"], a.ds, sysp["xN"], 0.1)
    run.set_fields(fields.to_physical(a.solver, wA), fields.to_physical(a.solver, wB))
    run.set_precision(a.precision)
    run.iterate(1)
    h = run.iterate(a.iterations)
    for i, F in enumerate(h["F"]):
        print(f"iteration {i + 1}: F = {F:.12f}")
    run.close()
    G.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
