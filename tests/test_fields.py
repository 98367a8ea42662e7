"""Host-side logic: seeded fields, the per-solver layout conventions of main()
(src/crysSCFT_sample.cpp:202-258) and the contour counts (:442-444)."""
import numpy as np
import pytest

from crysscft_sample_b200 import fields
from crysscft_sample_b200.scft import contour_counts
from oracle import scft_oracle as O


def test_seed_fields_are_deterministic_and_mirror_symmetric():
    a1, b1 = fields.seed_fields((16, 24, 32), 4.2, "FCC", seed=7)
    a2, b2 = fields.seed_fields((16, 24, 32), 4.2, "FCC", seed=7)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    for ax in range(3):
        assert np.array_equal(a1, np.flip(a1, axis=ax))
    a3, _ = fields.seed_fields((16, 24, 32), 4.2, "FCC", seed=8)
    assert not np.array_equal(a1, a3)


def test_gaussian_moments():
    z = fields.gaussian(1, 0, 200000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01


def test_bcc_shape_and_amplitude():
    wA, wB = fields.seed_fields((32, 32, 32), 4.2, "BCC", sigma=0.0)
    assert np.allclose(wA, -wB)
    assert 2.0 < wA.max() <= 6.0 + 1e-12  # A * (cc + cc + cc) <= 3A


@pytest.mark.parametrize("kind", ["P1", "3M", "PMMM"])
def test_layout_round_trip(kind):
    wA, _ = fields.seed_fields((16, 16, 32), 4.2)
    phy = fields.to_physical(kind, wA)
    assert np.array_equal(fields.from_physical(kind, phy, wA.shape), wA)


def test_layouts_follow_main():
    full = np.arange(8 * 8 * 8, dtype=float).reshape(8, 8, 8)
    assert np.array_equal(fields.to_physical("3M", full)[1, 2, 3], full[2, 4, 6])
    assert np.array_equal(fields.to_physical("PMMM", full)[1, 2, 3], full[1, 2, 3])
    assert fields.to_physical("PMMM", full).shape == (4, 4, 4)


@pytest.mark.parametrize("fA,ds,want", [(0.25, 0.01, (25, 75)), (0.25, 0.005, (50, 150)),
                                         (0.22, 0.005, (44, 156)), (0.2, 0.01, (20, 80))])
def test_contour_counts_truncate_like_the_reference(fA, ds, want):
    assert contour_counts(fA, ds) == want
    assert O.contour_counts(fA, ds) == want


def test_batch_config_is_seeded_and_in_range():
    from crysscft_sample_b200 import batch

    a = batch.batch_config(64)
    b = batch.batch_config(64)
    assert a == b and len(a) == 64
    for it in a:
        assert it["N"][0] // 2 in (16, 24, 32, 48, 64)
        assert 14.0 <= it["xN"] <= 30.0 and 0.2 <= it["fA"] <= 0.35 and 3.8 <= it["L"] <= 5.5
        assert it["phase"] in ("BCC", "FCC")
    assert len({it["N"] for it in a}) == 5
