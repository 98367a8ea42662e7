"""The configured-size fixtures (tests/golden/cfg_*.npz, made by make_golden_configs.py from
the reference build) are consistent: the reference's three solvers agree with each other
on the same symmetric fields, and a short rerun of the reference reproduces the start of
a stored history."""
import os

import numpy as np
import pytest

from oracle import ref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def test_fixtures_present():
    for name in ("cfg_bcc128_pmmm", "cfg_fcc128_pmmm", "cfg_bcc128_3m", "cfg_bcc128_p1", "cfg_bcc256_pmmm",
                 "cfg_bcc256_3m"):
        f = _load(name)
        assert np.all(np.isfinite(f["F"])) and f["idx"].size == 8192
        assert f["phiA"].shape == f["idx"].shape


@pytest.mark.parametrize("a,b,n", [("cfg_bcc128_3m", "cfg_bcc128_p1", 10), ("cfg_bcc128_pmmm", "cfg_bcc128_3m", 10),
                                   ("cfg_bcc256_pmmm", "cfg_bcc256_3m", 2)])
def test_reference_solvers_agree_in_fixtures(a, b, n):
    fa, fb = _load(a), _load(b)
    assert np.abs(fa["F"][:n] - fb["F"][:n]).max() < 1e-12 * np.abs(fa["F"][:n]).max()
    assert np.abs(fa["Q"][:n] - fb["Q"][:n]).max() < 1e-12 * np.abs(fa["Q"][:n]).max()


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_rerun_reproduces_fixture_start():
    import sys

    sys.path.insert(0, GOLDEN)
    import make_golden_configs as mk

    cfg = mk.CONFIGS["cfg_bcc128_3m"]
    a, b = mk.start_fields(cfg)
    out = ref.RefSolver(cfg["kind"], (cfg["N"],) * 3).scft_run(cfg["fA"], cfg["ds"], cfg["xN"], (cfg["L"],) * 3,
                                                                cfg["acc"], 2, a, b)
    want = _load("cfg_bcc128_3m")
    assert np.abs(out["F"] - want["F"][:2]).max() < 1e-13 * abs(want["F"][0])
