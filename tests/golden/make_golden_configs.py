"""Generate the configured-size fixtures tests/golden/cfg_*.npz from the reference itself.

The reference's own solvers and driver loop (compiled unmodified as
oracle/_ref/libscft_ref.so by oracle/Makefile, with the FFTW-API shim standing in for
FFTW) run the configured SCFT systems at full size.  Those runs take minutes of CPU
time, so the GPU tests compare against their stored results instead of rerunning them:

  per iteration: F, the four energy parts, max incompressibility, Q (all of them);
  after the last iteration: phiA, phiB, wA at 8192 seeded sample points of the
  physical grid (indices stored), plus the full-field sums of phiA and phiB.

Systems (driver loop src/crysSCFT_sample.cpp:440-508, seeded fields of fields.seed_fields):
  cfg_bcc128_pmmm   BCC, 128^3 full grid (PMMM on 64^3), L=4.2, fA=0.25, chiN=20,
                    ds=0.005 (Ns=200), lambda=0.1, 100 iterations
  cfg_fcc128_pmmm   FCC, 128^3 (PMMM on 64^3), L=5.0, fA=0.22, chiN=25, ds=0.005,
                    lambda=0.1, 100 iterations
  cfg_bcc128_3m     the BCC system with the 3m solver (64^3 even sub-lattice), 10 iterations
  cfg_bcc128_p1     the BCC system with P1 on the full 128^3 grid, 10 iterations
  cfg_bcc256_pmmm   the BCC system on a 256^3 full grid (PMMM on 128^3), 2 iterations
  cfg_bcc256_3m     the same with the 3m solver, 2 iterations

P1 on a 256^3 full grid needs (NsA+NsB+2) x 2 contour slices of 134 MB (54 GB) in the
reference's driver, more host memory than this generator assumes; the GPU test checks
it against the PMMM 256^3 run instead (same symmetric fields, the solvers agree).

Run from the repository root (needs the reference tree; all host cores are used):
    python tests/golden/make_golden_configs.py [name ...]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from crysscft_sample_b200 import fields  # noqa: E402
from oracle import ref  # noqa: E402

BCC = dict(phase="BCC", L=4.2, fA=0.25, xN=20.0, ds=0.005, acc=0.1)
FCC = dict(phase="FCC", L=5.0, fA=0.22, xN=25.0, ds=0.005, acc=0.1)

CONFIGS = {
    "cfg_bcc128_pmmm": dict(BCC, kind="PMMM", N=128, nstep=100),
    "cfg_fcc128_pmmm": dict(FCC, kind="PMMM", N=128, nstep=100),
    "cfg_bcc128_3m": dict(BCC, kind="3M", N=128, nstep=10),
    "cfg_bcc128_p1": dict(BCC, kind="P1", N=128, nstep=10),
    "cfg_bcc256_pmmm": dict(BCC, kind="PMMM", N=256, nstep=2),
    "cfg_bcc256_3m": dict(BCC, kind="3M", N=256, nstep=2),
}
NSAMPLE = 8192


def sample_indices(M: int, seed: int = 4242) -> np.ndarray:
    """Sorted, distinct sample points of a physical grid of M points."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(M, size=min(NSAMPLE, M), replace=False)).astype(np.int64)


def start_fields(cfg):
    N = (cfg["N"],) * 3
    wA, wB = fields.seed_fields(N, cfg["L"], cfg["phase"])
    return fields.to_physical(cfg["kind"], wA), fields.to_physical(cfg["kind"], wB)


def generate(name: str) -> None:
    cfg = CONFIGS[name]
    N = (cfg["N"],) * 3
    a, b = start_fields(cfg)
    R = ref.RefSolver(cfg["kind"], N)
    t0 = time.time()
    out = R.scft_run(cfg["fA"], cfg["ds"], cfg["xN"], (cfg["L"],) * 3, cfg["acc"], cfg["nstep"], a, b)
    idx = sample_indices(a.size)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        F=out["F"], parts=out["parts"], maxinc=out["maxinc"], Q=out["Q"], idx=idx,
        phiA=out["phiA"][idx], phiB=out["phiB"][idx], wA=out["wA"][idx],
        phiA_sum=np.array(np.sum(out["phiA"], dtype=np.longdouble), dtype=np.float64),
        phiB_sum=np.array(np.sum(out["phiB"], dtype=np.longdouble), dtype=np.float64),
        config=np.array(repr({k: v for k, v in cfg.items()})))
    print(f"{name}: {cfg['nstep']} iterations in {time.time() - t0:.1f} s, F[-1] = {out['F'][-1]:.12f}", flush=True)


def main(names):
    ref.build()
    ref.set_num_threads(os.cpu_count() or 1)
    for name in names or CONFIGS:
        generate(name)


if __name__ == "__main__":
    main(sys.argv[1:])
