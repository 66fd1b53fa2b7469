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
    assert (a.gpus, a.steps, a.warmup, a.impl, a.precision, a.workload) == (1, steps, warmup, "ours", "fp64",
                                                                            "string")
    assert a.warmup >= 3


def test_cpu_props_timing_bounds_the_sample():
    """The CPU legs time the oracle (test infrastructure) on a bounded sample:
    at least min_calls calls, at most max_calls."""
    import numpy as np
    m, D, N = (8, 8, 8), (2.0, 2.0, 2.0), 20
    wm = 0.5 * np.cos(2 * np.pi * np.arange(8) / 8)[:, None, None] * np.ones(m)
    t, n = bench.cpu_props_seconds(m, D, N, wm, np.zeros(m), 0.1, 0.8, 0.5, 1, threads=1, budget_s=0.0,
                                   max_calls=20, min_calls=3)
    assert n == 3 and t > 0
    t, n = bench.cpu_props_seconds(m, D, N, wm, np.zeros(m), 0.1, 0.8, 0.5, 1, threads=1, budget_s=60.0,
                                   max_calls=4)
    assert n == 4


def test_cpu_step_rate_matches_the_oracle_step():
    """cpu_step_rate advances q and q^dagger with the oracle's do_step; the
    step it times is the one props chains (same result as props' slice 1)."""
    import numpy as np

    import oracle as O
    m, D, N = (8, 8, 8), (2.0, 2.0, 2.0), 20
    wm = 0.5 * np.cos(2 * np.pi * np.arange(8) / 8)[:, None, None] * np.ones(m)
    rate, n = bench.cpu_step_rate(m, D, N, wm, np.zeros(m), 0.5, threads=1, budget_s=0.0, min_steps=2)
    assert n == 2 and rate > 0
    M = 512
    d = O.Density(m, D, N)
    w = np.zeros(6 * M)
    w[:M] = wm.ravel()
    d.props(w, N, 0.1, 0.8, 0.5, 1)
    s = O.Density(m, D, 2)
    s.prepare(1.0 / N, w[:2 * M])
    q1 = s.do_step(np.ones(2 * M), 0, 10, 10)
    np.testing.assert_allclose(q1[:M], d.q(0, 1), rtol=1e-14)
    np.testing.assert_allclose(q1[M:], d.q(1, 1), rtol=1e-14)


def test_alu_peak_is_sms_times_lanes_times_clock():
    # B200: 148 SMs at 1965 MHz: 74.4 TFLOP/s FP32 and 37.2 FP64 (non-tensor, nominal)
    assert bench.alu_peak_tflops("fp32", sms=148, sm_mhz=1965.0) == pytest.approx(74.4457, rel=1e-4)
    assert bench.alu_peak_tflops("fp64", sms=148, sm_mhz=1965.0) == pytest.approx(37.2229, rel=1e-4)
