"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference's own solvers and driver functions (compiled unmodified as
oracle/_ref/libscft_ref.so by oracle/Makefile, with the FFTW-API shim) produce
every array stored here.  The reference ships no tests or golden vectors, and
its README output needs an input file that is not available, so these
fixtures are the pinned outputs of the reference on seeded inputs:

  triplets.npz   one diffusion() call of each solver on a seeded random field
  contour.npz    solve_diffusion_equation (both directions) for each solver
  scft_cfg0.npz  100 iterations of the small BCC system (32^3 full grid, L=4.2,
                 fA=0.25, chiN=20, ds=0.01, lambda=0.1) for all three solvers:
                 per-iteration F, energy parts, max incompressibility, Q, and the
                 final phi fields of the PMMM run

Run from the repository root (needs the reference tree):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from crysscft_sample_b200 import fields  # noqa: E402
from oracle import ref  # noqa: E402

TRIPLET_CASES = [
    ("PMMM", (32, 32, 32), (4.2, 4.2, 4.2), 0.01),
    ("3M", (32, 16, 48), (4.2, 3.7, 5.1), 0.01),
    ("P1", (16, 24, 8), (4.2, 3.7, 5.1), 0.01),
]
CFG0 = dict(N=(32, 32, 32), L=4.2, fA=0.25, xN=20.0, ds=0.01, acc=0.1)


def case_key(kind, N):
    return f"{kind}_{N[0]}x{N[1]}x{N[2]}"


def main():
    ref.build()
    ref.set_num_threads(1)
    out = {}
    for kind, N, L, ds in TRIPLET_CASES:
        R = ref.RefSolver(kind, N)
        R.set_cell_para(L)
        R.set_contour_step(ds)
        rng = np.random.default_rng(12345)
        q = rng.standard_normal(R.space_size_phy)
        k = case_key(kind, N)
        out[k + "_in"] = q
        out[k + "_out"] = R.diffusion(q)
        out[k + "_cell"] = np.array(L)
        out[k + "_ds"] = np.array(ds)
    np.savez_compressed(os.path.join(HERE, "triplets.npz"), **out)

    out = {}
    for kind in ("PMMM", "3M", "P1"):
        N = (16, 16, 16)
        wA, _ = fields.seed_fields(N, 4.2)
        w = fields.to_physical(kind, wA).ravel()
        wds = np.exp(-0.01 / 2 * w)
        R = ref.RefSolver(kind, N)
        R.set_cell_para((4.2, 4.2, 4.2))
        R.set_contour_step(0.01)
        ones = np.ones(R.space_size_phy)
        out[kind + "_wds"] = wds
        out[kind + "_fwd"] = R.solve_diffusion_equation(ones, wds, 10, 1)
        out[kind + "_bwd"] = R.solve_diffusion_equation(ones, wds, 10, -1)
    np.savez_compressed(os.path.join(HERE, "contour.npz"), **out)

    out = {}
    N, L = CFG0["N"], CFG0["L"]
    wA, wB = fields.seed_fields(N, L, "BCC")
    out["wA_full"] = wA
    out["wB_full"] = wB
    for kind in ("PMMM", "3M", "P1"):
        R = ref.RefSolver(kind, N)
        r = R.scft_run(CFG0["fA"], CFG0["ds"], CFG0["xN"], (L, L, L), CFG0["acc"], 100,
                       fields.to_physical(kind, wA), fields.to_physical(kind, wB))
        for key in ("F", "parts", "maxinc", "Q"):
            out[f"{kind}_{key}"] = r[key]
        if kind == "PMMM":
            out["PMMM_phiA"] = r["phiA"]
            out["PMMM_phiB"] = r["phiB"]
            out["PMMM_wA_final"] = r["wA"]
    np.savez_compressed(os.path.join(HERE, "scft_cfg0.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
