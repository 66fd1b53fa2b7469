"""Runs the reference CUDA program (``oracle/_ref/scft_ref_*``, built by
``oracle/build_ref.sh``) on a seeded workload and times its string
iterations.  TEST INFRASTRUCTURE: used by the reference leg of ``bench.py``
and by the golden-fixture generator, never by the product.

The patched reference prints ``KSTART k t`` (CLOCK_MONOTONIC seconds) at the
start of every ``solve_field`` iteration (scft.cu:592-593).  After the
requested number of iterations has started, the run is stopped through the
reference's own graceful-stop path: SIGINT sets ``sigg=7`` (scft.cu:285-303),
the loop breaks at the end of the iteration (scft.cu:800-804) and the program
writes its outputs and exits.
"""
from __future__ import annotations

import os
import signal
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from scft_string_b200.configs import fields, input_dat, win_text  # noqa: E402


def binary_for(strn: int, nsterp: int = 4000, prelude: int = 5000) -> str:
    return os.path.join(HERE, "_ref", f"scft_ref_s{strn}_n{nsterp}_p{prelude}")


def time_iterations(cfg: dict, warmup: int, steps: int, timeout: float = 1500.0,
                    nsterp: int = 4000) -> dict:
    """Runs the reference on ``cfg`` until iteration warmup+steps has started
    and returns the wall time of iterations [warmup, warmup+steps)."""
    exe = binary_for(cfg["strn"], nsterp)
    if not os.path.exists(exe):
        return dict(unavailable=f"reference binary {os.path.basename(exe)} not built "
                                "(oracle/build_ref.sh needs the reference sources)")
    wm, wp = fields(cfg)
    stamps = {}
    props_lines = 0
    props_in_window = 0
    kcur = -1
    t0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input.dat"), "w") as fh:
            fh.write(input_dat(cfg))
        for ii in range(cfg["strn"]):
            with open(os.path.join(d, f"win{ii}"), "w") as fh:
                fh.write(win_text(wm[ii], wp[ii]))
        proc = subprocess.Popen([exe], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                text=True, bufsize=1)
        stopped = False
        try:
            for line in proc.stdout:
                if line.startswith("PROPS"):
                    props_lines += 1
                    if warmup <= kcur < warmup + steps:
                        props_in_window += 1
                elif line.startswith("KSTART"):
                    _, k, t = line.split()
                    stamps[int(k)] = float(t)
                    kcur = int(k)
                    if int(k) >= warmup + steps and not stopped:
                        proc.send_signal(signal.SIGINT)
                        stopped = True
                if time.time() - t0 > timeout and not stopped:
                    proc.send_signal(signal.SIGINT)
                    stopped = True
            proc.wait(timeout=600)
        finally:
            if proc.poll() is None:
                proc.kill()
                proc.wait()
    if warmup + steps not in stamps or warmup not in stamps:
        return dict(unavailable=f"reference stopped before iteration {warmup + steps} "
                                f"(rc={proc.returncode})")
    sec = stamps[warmup + steps] - stamps[warmup]
    return dict(seconds=sec, iters=steps, iters_per_s=steps / sec, props_lines=props_lines,
                props_in_window=props_in_window, wall=time.time() - t0)
