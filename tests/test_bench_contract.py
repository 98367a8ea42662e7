"""bench.py's reference arm runs on CPU and prints one JSON line with the keys the
benchmark contract requires (the GPU arm is exercised on the GPU box)."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_arm_prints_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "32",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["config"]["workload"]


def test_reference_arm_nonzero_rank_exits_quietly():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "32",
                          "--steps", "1"], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, RANK="1", WORLD_SIZE="2"))
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_hbm_peak_reads_measured_file_or_falls_back(tmp_path, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    peak, src = bench.hbm_peak()
    assert peak > 0 and src in ("measured", "fallback")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.hbm_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6500.5}))
    assert bench.hbm_peak() == (6500.5, "measured")
    assert isinstance(bench.cpu_model(), str) and bench.cpu_model()
