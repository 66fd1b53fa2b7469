"""CPU checks of the benchmark's helpers (no GPU, no library calls): the peak
and traffic lookups that the roofline object of the JSON line is built from,
and the command-line defaults the driver relies on."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_peaks_measured_and_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6445.6, "bf16_tflops": 1590}))
    assert bench.peaks() == (6445.6, "measured")
    (tmp_path / "MEASURED_PEAKS.json").write_text("{not json")
    assert bench.peaks() == (6650.0, "fallback")


def test_profiled_traffic_reads_the_committed_summary():
    t = bench.profiled_traffic()
    assert t is not None and 8.39e6 < t < 1e8   # above the 8.39 MB algorithmic bytes of a 64^3 step


@pytest.mark.parametrize("argv,steps,warmup", [([], 20, 3), (["--steps", "5", "--warmup", "4"], 5, 4)])
def test_defaults(monkeypatch, argv, steps, warmup):
    monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
    a = bench.parse()
    assert (a.gpus, a.steps, a.warmup, a.impl, a.precision, a.workload) == (1, steps, warmup, "ours", "fp32",
                                                                            "string")
    assert a.warmup >= 3
