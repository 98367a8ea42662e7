"""Checkpoint file format (crysscft_sample_b200.checkpoint): round trip of the header and
the fields, and rejection of foreign or incomplete files.  CPU only."""
import numpy as np
import pytest

from crysscft_sample_b200 import checkpoint


def _meta():
    return {"kind": "PMMM", "grid_log": [32, 32, 32], "cell": [4.2, 4.2, 4.2, 0, 0, 0], "fA": 0.25, "ds": 0.01,
            "xN": 20.0, "acceptance": 0.1, "iterations": 7, "precision": "fp64", "mixing": ["anderson", 8, 0.5],
            "translational_part": None, "anisotropic": False}


def test_round_trip(tmp_path):
    rng = np.random.default_rng(8)
    f = {k: rng.standard_normal(4096) for k in ("wA", "wB", "phiA", "phiB")}
    p = tmp_path / "c.npz"
    checkpoint.write(p, _meta(), f)
    meta, g = checkpoint.read(p)
    assert meta == _meta()
    for k in f:
        assert np.array_equal(f[k], g[k])


def test_rejects_foreign_and_incomplete(tmp_path):
    p = tmp_path / "x.npz"
    np.savez(p, header=np.frombuffer(b'{"format": "other"}', dtype=np.uint8), wA=np.zeros(1), wB=np.zeros(1),
             phiA=np.zeros(1), phiB=np.zeros(1))
    with pytest.raises(ValueError):
        checkpoint.read(p)
    m = _meta()
    del m["ds"]
    with pytest.raises(ValueError):
        checkpoint.write(tmp_path / "y.npz", m, {k: np.zeros(4) for k in ("wA", "wB", "phiA", "phiB")})
    with pytest.raises(ValueError):
        checkpoint.write(tmp_path / "z.npz", _meta(), {"wA": np.zeros(4), "wB": np.zeros(5), "phiA": np.zeros(4),
                                                        "phiB": np.zeros(4)})
