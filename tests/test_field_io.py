"""The reference's text field format (src/crysSCFT_sample.cpp:271-292): our writer produces
the same bytes as the reference's output_fields, and our reader reads what the
reference writes (and vice versa)."""
import ctypes
import os

import numpy as np
import pytest

from crysscft_sample_b200 import fields
from oracle import ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@needs_ref
def test_writer_matches_reference_bytes(tmp_path):
    rng = np.random.default_rng(5)
    arrs = [rng.standard_normal(512) * s for s in (1e-3, 1.0, 30.0, 1e5)]
    arrs[0][0] = 0.0
    ours, theirs = str(tmp_path / "ours.txt"), str(tmp_path / "theirs.txt")
    fields.write_fields_text(ours, *arrs)
    p = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in arrs]
    ref.lib().ref_output_fields(*p, 512, theirs.encode())
    assert open(ours).read() == open(theirs).read()


@needs_ref
def test_reader_round_trips_with_reference(tmp_path):
    rng = np.random.default_rng(6)
    arrs = [rng.standard_normal(300) for _ in range(4)]
    path = str(tmp_path / "full.txt")
    fields.write_fields_text(path, *arrs, precision=17)
    got = fields.read_fields_text(path, 300)
    for a, b in zip(arrs, got):
        assert np.array_equal(a, b)
    back = [np.zeros(300) for _ in range(4)]
    p = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in back]
    ref.lib().ref_input_fields(*p, 300, path.encode())
    for a, b in zip(arrs, back):
        assert np.array_equal(a, b)


def test_reader_rejects_short_files(tmp_path):
    path = str(tmp_path / "short.txt")
    open(path, "w").write("1 2 3 4\n")
    with pytest.raises(ValueError):
        fields.read_fields_text(path, 2)
