#!/usr/bin/env python3
"""Benchmark: string iterations per second of the SCFT string method.

Workload: the 16-replica 64^3 string (N=128, chiN=14, f=0.45, phidb=0.85,
D=5, fixed ends; ens=2, the reference default), seeded synthetic fields
(scft_string_b200.configs.STRING_64).  One step = one iteration of the
reference's solve_field loop (scft.cu:592-806): inner W+ relaxation and props
of every replica, residuals, spline tangent projection, mixing and equal-arc
redistribution.  Each rank runs its own copy of the string (replicas only, no
collective on the data path); value = steps of all ranks / max-rank device time.

The default timed arm is the batched FP64 path: the reference's arithmetic,
so its ratio to the reference arm compares like with like.  The batched FP32
path (the metric's "fused FP32") and the plain FP64 path (one replica at a
time) are timed on the same iterations and reported beside it, with the FP32
path's errors against FP64 at identical fields.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp32|fp64] [--plain]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "String iters/s @ RMS err≤1e-5, batched fused FP32 vs plain FP64 on 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp32", "fp64"],
                    help="propagator arithmetic of the timed arm (fp64: the reference's; the other precision "
                         "and plain FP64 run on the same window beside it)")
    ap.add_argument("--plain", action="store_true", help="one replica at a time")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--workload", default="string",
                    choices=["string", "uneven24", "mixed128", "adjoint96", "tolerance"],
                    help="uneven24: the 24 independent solves of mixed grids and N, run concurrently; "
                         "tolerance: the string run to RMS error --tol (time to the metric's error clause)")
    ap.add_argument("--switch", type=float, default=3e-5,
                    help="tolerance: errtot at which the FP32 iterations hand the string to FP64")
    ap.add_argument("--max-iters", type=int, default=4000,
                    help="tolerance: string iteration cap (the reference's nsterp, scft.cu:1102)")
    ap.add_argument("--case", default="string64", choices=["string64", "plain32"],
                    help="tolerance: the 16-replica 64^3 string, or the 32^3 single-replica workload")
    ap.add_argument("--compare", action="store_true",
                    help="tolerance: run FP32 -> FP64 and FP64 only, and compare their final F")
    ap.add_argument("--time-limit", type=float, default=0.0,
                    help="tolerance: stop (reached = false) after this many wall seconds (0: none)")
    ap.add_argument("--tol", type=float, default=1e-5, help="uneven24: RMS residual target")
    ap.add_argument("--start", default="lamellar", choices=["lamellar", "hex"],
                    help="adjoint96: start field of the saddle point search")
    ap.add_argument("--iters", type=int, default=5000, help="uneven24: Anderson iteration cap per solve")
    ap.add_argument("--serial-fp64", action="store_true",
                    help="uneven24: also run the solves one at a time on the plain FP64 path")
    ap.add_argument("--profile-round", type=int, default=0, metavar="R",
                    help="profiling mode: one batched props round of R replicas of the workload, then exit")
    return ap.parse_args()


def profile_round(a, cfg):
    """One batched props round (prepare, 4 launches per contour step, densities)
    of the first R replicas of the workload: the unit the ncu captures in
    profiles/ are taken on."""
    import scft_string_b200 as S
    from scft_string_b200.configs import fields
    c = dict(cfg)
    c["strn"] = a.profile_round
    wm, wp = fields(c)
    ctx = S.StringSolver(c, precision=a.precision, batched=not a.plain)
    for ii in range(c["strn"]):
        ctx.set_fields(ii, wm[ii], wp[ii])
    ctx.solve_field0_all(2, 0.0)
    print(json.dumps({"profile_round": c["strn"], "precision": a.precision, **ctx.stats()}))
    return 0


def dist_env():
    from scft_string_b200 import dist as D
    return D.env()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 8:
                    rows.append(t)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = sorted(float(r[0]) for r in rows if r[0].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def alu_peak_tflops(precision, sms=None, sm_mhz=None):
    """Nominal non-tensor peak of the precision's pipe: SMs x FMA lanes per SM
    (128 FP32, 64 FP64 on sm_100) x 2 flops x the maximum SM clock.
    MEASURED_PEAKS.json has no FP32 or FP64 ALU figure, so this one is
    computed, not measured; the SM count comes from the device (148 when none
    is visible) and the clock from MEASURED_PEAKS.json (1965 MHz otherwise)."""
    if sms is None:
        sms = 148
        try:
            import torch
            if torch.cuda.is_available():
                sms = torch.cuda.get_device_properties(0).multi_processor_count
        except Exception:
            pass
    if sm_mhz is None:
        sm_mhz = 1965.0
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
                sm_mhz = float(json.load(fh).get("sm_max_mhz", sm_mhz))
        except (OSError, ValueError):
            pass
    lanes = 128 if precision == "fp32" else 64
    return sms * lanes * 2 * sm_mhz * 1e6 / 1e12


def profiled_traffic(precision="fp32"):
    """DRAM bytes per replica contour step from the committed ncu summary of
    the precision's step kernels (None when no capture was summarised)."""
    path = os.path.join(ROOT, "profiles", "step_traffic.txt")
    key = "dram_bytes_per_replica_step" if precision == "fp32" else f"dram_bytes_per_replica_step_{precision}"
    try:
        with open(path) as fh:
            for line in fh:
                t = line.split()
                if len(t) >= 2 and t[0] == key:
                    return float(t[1])
    except OSError:
        pass
    return None


def cpu_props_seconds(m, D, N, wm, wp, alpha, phidb, f, ens, threads, budget_s=10.0, max_calls=20, min_calls=1):
    """Seconds per FP64 oracle props call (the reference algorithm restated in
    C, OpenMP over grid points) at the fields wm, wp on `threads` host threads:
    at least min_calls calls, then more while the time budget lasts and fewer
    than max_calls were made.  Returns (seconds per call, calls made)."""
    import numpy as np

    import oracle as O
    O.set_threads(threads)
    M = int(np.prod(m))
    d = O.Density(m, D, N)
    w = np.zeros(6 * M)
    w[:M], w[M:2 * M] = np.ravel(wm), np.ravel(wp)
    fr = round(N * f) / N
    t0 = time.time()
    n = 0
    while n < min_calls or (time.time() - t0 < budget_s and n < max_calls):
        d.props(w, N, alpha, phidb, fr, ens)
        n += 1
    return (time.time() - t0) / n, n


def cpu_step_rate(m, D, N, wm, wp, f, threads, budget_s=10.0, min_steps=2, max_steps=50):
    """Contour steps per second of the FP64 oracle's Richardson step (q and
    q^dagger advanced by ds, as do_step, density.h:129-220) on `threads` host
    threads, over a bounded number of steps.  The density sum is not timed, and
    only the step's scratch is allocated, not the N+1 slices of a props store
    (6.7 GB at 128^3, N = 200).  Returns (steps per second, steps timed)."""
    import numpy as np

    import oracle as O
    O.set_threads(threads)
    M = int(np.prod(m))
    d = O.Density(m, D, 2)
    d.prepare(1.0 / N, np.concatenate([np.ravel(wm), np.ravel(wp)]))
    n1 = int(round(N * f))
    q = np.ones(2 * M)
    t0 = time.time()
    n = 0
    while n < min_steps or (time.time() - t0 < budget_s and n < max_steps):
        q = d.do_step(q, n % N, n1, N - n1)
        n += 1
    return n / (time.time() - t0), n


def cpu_baseline(cfg, props_per_iter):
    """The FP64 oracle (the reference algorithm restated in C, OpenMP over
    grid points) timed on the host cores: a bounded sample of props calls of
    one replica of the workload, scaled to string iterations by the props
    calls per replica and iteration counted in the timed window."""
    import oracle as O
    from scft_string_b200.configs import fields
    cores = os.cpu_count() or 1
    wm, wp = fields(cfg)
    args = (cfg["m"], cfg["D"], cfg["N"], wm[1], wp[1], cfg.get("alpha", 0.1), cfg["phidb"], cfg["f"], cfg["ens"])
    tp, n = cpu_props_seconds(*args, threads=cores, budget_s=10.0, max_calls=20, min_calls=3)
    # the same on one core (one or two props calls)
    tp1, _ = cpu_props_seconds(*args, threads=1, budget_s=8.0, max_calls=2)
    O.set_threads(cores)
    m = cfg["m"]
    return {"value": 1.0 / (props_per_iter * cfg["strn"] * tp), "unit": "string iters/s",
            "value_1core": 1.0 / (props_per_iter * cfg["strn"] * tp1), "props_s_1core": tp1,
            "cores": cores, "kind": "port",
            "sample": f"{n} props calls of one replica ({m[0]}x{m[1]}x{m[2]}, N={cfg['N']}, FP64, {cores} "
                      f"threads), {tp:.3f} s each; rate = 1/(props per iteration x replicas x that time) "
                      f"with {props_per_iter:.2f} props per replica per iteration, counted in the timed "
                      "window; the string coupling (O(replicas x M) per iteration) is not in the sample",
            "contour_steps_per_s": cfg["N"] / tp}


def run_uneven(a):
    """The uneven batch: every solve has its own context and stream, a host
    thread per solve drives its Anderson iteration, the GPU runs them
    concurrently.  Reports aggregate contour steps per second."""
    import concurrent.futures as cf

    import torch

    import scft_string_b200 as S
    from scft_string_b200.configs import noise_fields, uneven_batch
    solves = uneven_batch()
    torch.cuda.set_device(0)

    def make(c, prec):
        ctx = S.Context(c["m"], c["D"], c["N"], chi=c["chi"], f=c["f"], phidb=c["phidb"], ens=c["ens"],
                        alpha=c["alpha"], strn=1, dostring=0, precision=prec, batched=True)
        wm, wp = noise_fields(c)
        ctx.set_fields(0, wm, wp)
        return ctx

    def solve(ctx):
        n, err = ctx.anderson_solve(0, maxIter=a.iters, tol=a.tol, nhist=12, lam=0.1)
        return n, err, ctx.stats()["contour_steps"]

    ctxs = [make(c, a.precision) for c in solves]
    for c in ctxs:  # warm-up: graph capture and first launches
        c.props(0)
        c.reset_stats()
    torch.cuda.synchronize()
    t0 = time.time()
    with cf.ThreadPoolExecutor(max_workers=len(ctxs)) as ex:
        res = list(ex.map(solve, ctxs))
    wall = time.time() - t0
    steps = sum(r[2] for r in res)
    b = 4 if a.precision == "fp32" else 8
    algo = sum(r[2] * 8 * c["m"][0] * c["m"][1] * c["m"][2] * b for r, c in zip(res, solves))
    peak, peak_kind = peaks()
    line = {"metric": "aggregate contour steps/s, uneven batch of 24 solves to RMS residual "
                      f"{a.tol:g}", "value": steps / wall, "unit": "contour steps/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32" if a.precision == "fp32" else "f64",
            "data": "synthetic (seeded fields, scft_string_b200.configs.uneven_batch)",
            "config": {"workload": "uneven24: 8x48^3, 10x64^3, 6x96^3, N in {64..256}, ens=2",
                       "solver": "Anderson (FP64 least squares), one context and stream per solve"},
            "wall_s": wall, "iterations": [r[0] for r in res], "residuals": [r[1] for r in res],
            "converged": sum(1 for r in res if r[1] <= a.tol), "iteration_cap": a.iters,
            "roofline": {"bound": "hbm", "achieved": algo / wall / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / wall / 1e9 / peak, "peak_kind": peak_kind,
                         "note": "8 M b algorithmic bytes per contour step, wall time of the whole batch"}}
    cores = os.cpu_count() or 1
    c64 = next(c for c in solves if c["m"][0] == 64)
    wm0, wp0 = noise_fields(c64)
    rate, n = cpu_step_rate(c64["m"], c64["D"], c64["N"], wm0, wp0, c64["f"], cores, budget_s=10.0)
    line["cpu_baseline"] = {"contour_steps_per_s": rate, "cores": cores, "kind": "port",
                            "sample": f"{n} Richardson steps of one 64^3 solve of the batch (N={c64['N']}, FP64, "
                                      f"{cores} threads); the density sum is not timed"}
    if a.serial_fp64:
        s64 = 0
        w64 = 0.0
        for c in solves:
            ctx = make(c, "fp64")
            ctx.props(0)
            ctx.reset_stats()
            torch.cuda.synchronize()
            t1 = time.time()
            n, err, st = solve(ctx)
            w64 += time.time() - t1
            s64 += st
            ctx.close()
        line["serial_fp64"] = {"wall_s": w64, "contour_steps_per_s": s64 / w64}
        line["speedup_vs_serial_fp64_wall"] = w64 / wall
    print(json.dumps(line))
    return 0


def tolerance_run(a, cfg, precision):
    """One run of the reference's solve_field iterations (scft.cu:592-806;
    its loop never stops on the error, scft.cu:563) until errtot =
    sqrt(mean errs3^2) (scft.cu:764-765) <= a.tol, a.max_iters or
    a.time_limit, after the W+ prelude (scft.cu:1105).
      precision fp32: FP32 batched iterations until errtot <= a.switch (or no
        1 % progress over 200 iterations), then the fields go device to device
        to an FP64 batched context that continues the same run (same k) to
        a.tol; F per replica from a final FP64 FreeE;
      precision fp64: FP64 batched from the start.
    Device time per phase (CUDA events on each context's stream), the errtot
    history, F per replica, and -- at the hand-over -- the FP32 errors against
    FP64 at identical fields."""
    import numpy as np

    import scft_string_b200 as S
    from scft_string_b200.configs import fields
    strn, M = cfg["strn"], int(np.prod(cfg["m"]))
    wm, wp = fields(cfg)
    t_wall = time.time()
    first = S.StringSolver(cfg, precision=precision, batched=True)
    for ii in range(strn):
        first.set_fields(ii, wm[ii], wp[ii])
    first.autotune()
    first.timer_mark(0)
    first.solve_field0_all(5000, 1e-4)  # prelude, scft.cu:1105
    first.timer_mark(1)
    prelude_ms = first.timer_elapsed_ms(0, 1)
    hist = []
    out = {"workload": "tolerance: " + cfg["name"], "tol": a.tol, "mode": precision, "max_iters": a.max_iters,
           "prelude_s": prelude_ms / 1e3}

    def phase(ctx, k0, stop_tol, stall):
        ctx.string_resume(k0, a.max_iters, 1e-3)
        ctx.reset_stats()
        ctx.timer_mark(2)
        best, best_k, k = float("inf"), k0, k0
        while k < a.max_iters:
            r = ctx.string_step()
            hist.append((r["k"], r["errtot"]))
            k = r["k"] + 1
            if r["errtot"] < 0.99 * best:
                best, best_k = r["errtot"], k
            if r["errtot"] <= stop_tol or (stall and k - best_k >= 200):
                break
            if a.time_limit > 0 and time.time() - t_wall > a.time_limit:
                out["time_limited"] = True
                break
        ctx.timer_mark(3)
        st = ctx.stats()
        return k, dict(iters=k - k0, seconds=ctx.timer_elapsed_ms(2, 3) / 1e3, errtot_end=hist[-1][1] if hist else None,
                       props_per_replica_iter=st["props_calls"] / max(1, (k - k0) * strn),
                       contour_steps_per_s=st["contour_steps"] / max(1e-30, st["props_seconds"]))

    if precision == "fp32":
        k, p32 = phase(first, 0, a.switch, True)
        out["phase_fp32"] = p32
        W = [np.ascontiguousarray(first.get_fields(ii)) for ii in range(strn)]
        # FP32 errors against FP64 at the hand-over fields
        one64 = S.StringSolver(dict(cfg, strn=1), precision="fp64")
        one32 = S.StringSolver(dict(cfg, strn=1), precision="fp32")
        dF, dq, dr, dd = [], [], [], []
        for w in W:
            F64, q64, r64 = f_per_chain(one64, cfg, w)
            c64, _, _ = one64.get_conc(0)
            F32, q32, r32 = f_per_chain(one32, cfg, w)
            c32, _, _ = one32.get_conc(0)
            d64 = cfg["chi"] * (c64[M:2 * M] - c64[:M]) - 2 * w[:M]
            d32 = cfg["chi"] * (c32[M:2 * M] - c32[:M]) - 2 * w[:M]
            dF.append(abs(F32 - F64))
            dq.append(abs(q32 - q64) / max(1e-300, abs(q64)))
            dr.append(float(np.abs(r32 - r64).max()))
            dd.append(float(np.sqrt(np.mean((d32 - d64) ** 2))))
        one64.close()
        one32.close()
        out["fp32_errors_at_handover"] = {"k": k, "F_per_chain": dF, "lnQ_rel": dq, "rhoA_maxabs": dr,
                                          "exchange_residual_rms_diff": dd}
        second = S.StringSolver(cfg, precision="fp64", batched=True)
        second.autotune()
        second.copy_fields_from(first)
        first.close()
        if not out.get("time_limited"):
            k, p64 = phase(second, k, a.tol, False)
            out["phase_fp64"] = p64
        last = second
    else:
        k, p64 = phase(first, 0, a.tol, False)
        out["phase_fp64"] = p64
        last = first
    fe = last.free_energy()
    last.close()
    out["reached"] = bool(hist and hist[-1][1] <= a.tol)
    out["iterations"] = k
    out["time_to_tol_s"] = sum(out[p]["seconds"] for p in ("phase_fp32", "phase_fp64") if p in out)
    out["time_to_tol_with_prelude_s"] = out["time_to_tol_s"] + out["prelude_s"]
    out["iters_per_s"] = k / max(1e-30, out["time_to_tol_s"])
    out["F_per_replica_fp64"] = list(fe["FEs"])
    out["errtot_history"] = hist[::10] + hist[-1:]
    out["wall_s"] = time.time() - t_wall
    return out


def run_tolerance(a):
    """Time to the metric's error clause (tolerance_run) on the 16-replica 64^3
    string, or on the 32^3 single-replica workload (--case plain32).  With
    --compare, both the FP32 -> FP64 run and the FP64-only run, and the
    difference of their final F per replica."""
    import torch

    from scft_string_b200.configs import PLAIN_32, STRING_64
    torch.cuda.set_device(0)
    cfg = dict(STRING_64 if a.case == "string64" else PLAIN_32)
    if a.compare:
        runs = {p: tolerance_run(a, cfg, p) for p in ("fp32", "fp64")}
        F32, F64 = runs["fp32"]["F_per_replica_fp64"], runs["fp64"]["F_per_replica_fp64"]
        out = {"workload": "tolerance: " + cfg["name"], "fp32_then_fp64": runs["fp32"], "fp64_only": runs["fp64"],
               "F_diff_per_chain": [abs(x - y) for x, y in zip(F32, F64)],
               "time_ratio_fp64_only_over_mixed": runs["fp64"]["time_to_tol_s"] / max(1e-30, runs["fp32"]["time_to_tol_s"])}
    else:
        out = tolerance_run(a, cfg, a.precision)
    print(json.dumps(out))
    return 0


def f_per_chain(ctx, c, W):
    """props at fields W (2M) of replica 0 and F = -lnQ + <chi pA pB - wA pA - wB pB>."""
    import numpy as np
    M = ctx.M
    ctx.set_fields_2m(0, np.ascontiguousarray(W))
    ctx.props(0)
    conc, lnQ, _ = ctx.get_conc(0)
    pA, pB = conc[:M], conc[M:2 * M]
    wa, wb = W[:M] + W[M:], W[M:] - W[:M]
    return -lnQ + np.mean(c["chi"] * pA * pB - wa * pA - wb * pB), lnQ, pA


def run_mixed128(a):
    """128^3, N=200, 8 replicas: FP64 and FP32 from the same start; errors of the
    FP32 path at identical fields (lnQ, F, rhoA, errtot) and both throughputs."""
    import numpy as np
    import torch

    import scft_string_b200 as S
    from scft_string_b200.configs import MIXED_128, gyroid_fields
    torch.cuda.set_device(0)
    c = dict(MIXED_128)
    wm, wp = gyroid_fields(c)
    out = {"workload": c["name"]}
    W64 = None
    for prec in ("fp64", "fp32"):
        ctx = S.StringSolver(c, precision=prec, batched=True)
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        ctx.solve_field0_all(30, 0.0)
        ctx.string_begin(4000, 1e-3)
        ctx.string_step()  # k = 0 carries FreeE
        ctx.reset_stats()
        ctx.timer_mark(0)
        reps = [ctx.string_step() for _ in range(a.steps)]
        ctx.timer_mark(1)
        st = ctx.stats()
        out[prec] = {"iters_per_s": a.steps / (ctx.timer_elapsed_ms(0, 1) / 1e3),
                     "contour_steps_per_s": st["contour_steps"] / st["props_seconds"],
                     "errtot": [r["errtot"] for r in reps]}
        if prec == "fp64":
            W64 = [ctx.get_fields(ii) for ii in range(c["strn"])]
        ctx.close()
    # FP32 errors at the FP64 fields, replica by replica
    dF, dQ, drho = [], [], []
    one64 = S.StringSolver(dict(c, strn=1), precision="fp64")
    one32 = S.StringSolver(dict(c, strn=1), precision="fp32")
    for W in W64:
        F64, q64, r64 = f_per_chain(one64, c, W)
        F32, q32, r32 = f_per_chain(one32, c, W)
        dF.append(abs(F32 - F64))
        dQ.append(abs(q32 - q64) / abs(q64))
        drho.append(float(np.abs(r32 - r64).max()))
    e64 = np.array(out["fp64"]["errtot"])
    e32 = np.array(out["fp32"]["errtot"])
    out["fp32_error"] = {"F_per_chain_max": max(dF), "lnQ_rel_max": max(dQ), "rhoA_maxabs": max(drho),
                         "errtot_rel_max": float(np.max(np.abs(e32 - e64) / e64))}
    out["fp32_speedup"] = out["fp32"]["contour_steps_per_s"] / out["fp64"]["contour_steps_per_s"]
    cores = os.cpu_count() or 1
    rate, n = cpu_step_rate(c["m"], c["D"], c["N"], wm[0], wp[0], c["f"], cores, budget_s=15.0)
    out["cpu_baseline"] = {"contour_steps_per_s": rate, "cores": cores, "kind": "port",
                           "sample": f"{n} Richardson steps of one replica (128^3, FP64, {cores} threads); "
                                     "the density sum is not timed"}
    print(json.dumps(out))
    return 0


def run_adjoint96(a):
    """64x64x96, N=160 single replica: converged saddle point (Anderson), box
    stress from the FP64 and FP32 adjoints against central differences of
    re-converged FP64 free energies (h = 1e-4), dF/dchiN likewise, dF/df with a
    continuous A fraction against one-sided differences, then variable-cell
    relaxation to |stress| <= 1e-6."""
    import numpy as np
    import torch

    import scft_string_b200 as S
    from scft_string_b200.configs import ADJOINT_96, hex_fields, lamellar_fields
    torch.cuda.set_device(0)
    c = dict(ADJOINT_96)
    t0 = time.time()
    hex_note = None
    if a.start == "hex":
        # The stated start, 0.5 chiN sum_j cos(G_j.r), puts |W-| up to 1.5 chiN,
        # three times the self-consistent range |W-| <= chiN/2; simple, pressure
        # and Anderson mixing all diverge from it (W+ runs away).  The saddle is
        # sought from the same pattern at 0.2 of that amplitude.
        wm, wp = hex_fields(c)
        wm = 0.2 * wm
    else:
        # Lamellae along z (one period = Lz): the same grid, box, N, chiN and f;
        # a 1-D saddle that Anderson mixing converges to 1e-9.  The hexagonal
        # start is not commensurate with the square x-y cross-section and its
        # cylinders relax slowly (residual 1.8e-4 after 6000 iterations).
        wm, wp = lamellar_fields(c)
        hex_note = "hexagonal start: residual 1.8e-4 after 6000 Anderson iterations (not converged)"

    def converged(D, chi, prec="fp64", W0=None, f=None):
        cc = dict(c, D=tuple(D), chi=chi)
        if f is not None:  # continuous A fraction
            cc.update(f=f, fcont=1)
        ctx = S.StringSolver(cc, precision=prec)
        if W0 is None:
            ctx.set_fields(0, wm[0], wp[0])
        else:
            ctx.set_fields_2m(0, np.ascontiguousarray(W0))
        n, err = ctx.anderson_solve(0, maxIter=6000 if W0 is None else 3000, tol=1e-9, nhist=12, lam=0.1)
        F, _, _ = f_per_chain(ctx, cc, ctx.get_fields(0))
        return ctx, F, err, n

    D0 = np.array(c["D"])
    ctx, F0, err0, n0 = converged(D0, c["chi"])
    W = ctx.get_fields(0)
    _, dF64 = ctx.stress(0)
    _, dF64ck, bytes64 = ctx.stress_ckpt(0, 13)   # q kept every 13 contour steps
    c32 = S.StringSolver(c, precision="fp32")
    c32.set_fields_2m(0, np.ascontiguousarray(W))
    _, dF32, bytes32 = c32.stress_ckpt(0, 13)
    c32.close()
    store32 = (c["N"] + 1) * 2 * ctx.M * 4
    h = 1e-4
    fd = []
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        cp, Fp, _, _ = converged(D0 + e, c["chi"], W0=W)
        cp.close()
        cm, Fm, _, _ = converged(D0 - e, c["chi"], W0=W)
        cm.close()
        fd.append((Fp - Fm) / (2 * h))
    dchi = ctx.dF_dchi(0)
    cp, Fcp, _, _ = converged(D0, c["chi"] + h, W0=W)
    cp.close()
    cm, Fcm, _, _ = converged(D0, c["chi"] - h, W0=W)
    cm.close()
    fdc = (Fcp - Fcm) / (2 * h)
    # dF/df with a continuous A fraction: N f = 64 lies on a step boundary, so the
    # adjoint gives the right derivative; second-order one-sided differences
    f0 = c["f"]
    cf0, Ff0, _, _ = converged(D0, c["chi"], W0=W, f=f0)
    dFdf = cf0.dF_df(0)[1]
    cf32 = S.StringSolver(dict(c, fcont=1), precision="fp32")
    cf32.set_fields_2m(0, np.ascontiguousarray(cf0.get_fields(0)))
    dFdf32 = cf32.dF_df(0)[1]
    cf32.close()
    cf0.close()
    Ff = [Ff0]
    for k in (1, 2):
        ck_, Fk, _, _ = converged(D0, c["chi"], W0=W, f=f0 + k * h)
        ck_.close()
        Ff.append(Fk)
    fdf = (-3 * Ff[0] + 4 * Ff[1] - Ff[2]) / (2 * h)
    relax = None
    if err0 < 1e-6:  # relax from a converged saddle only
        n, st, box = ctx.relax_cell(0, maxOuter=20, inner=0, stressTol=1e-6, gamma=2.0)
        relax = {"rounds": n, "final_stress": list(st), "box": list(box)}
    out = {"workload": c["name"], "start": a.start, "hex_note": hex_note, "saddle_residual": err0, "anderson_iters": n0, "F": F0,
           "dF_dL_fp64_adjoint": list(dF64), "dF_dL_fp32_adjoint": list(dF32), "dF_dL_fd": fd,
           "dF_dL_fp32_vs_fp64_rel": float(np.max(np.abs(dF32 - dF64)) / max(1e-30, np.max(np.abs(dF64)))),
           "dF_dL_fp64_ckpt13_vs_full": float(np.max(np.abs(dF64ck - dF64))),
           "ckpt13_bytes_fp32": bytes32, "full_store_bytes_fp32": store32,
           "dF_dchi_closed_form": dchi, "dF_dchi_fd": fdc,
           "dF_df_fp64_adjoint": dFdf, "dF_df_fp32_adjoint": dFdf32, "dF_df_fd_one_sided": fdf,
           "relax": relax,
           "checkpointing": "FP32 adjoint with q, q^dagger kept every 13 contour steps (scft_stress_ckpt)",
           "wall_s": time.time() - t0}
    print(json.dumps(out))
    return 0


def run_ours(a, cfg, rank, world, dev):
    """Iterations k = W..W+K-1 of the string after the W+ prelude and W warm-up
    iterations, three times over the same window:
      value  device-resident fields, timed with CUDA events;
      e2e    the same iterations again from a host copy of the fields at k = W
             (scft_string_resume), with every replica's fields copied in from
             pinned host memory and back out in every iteration;
      cmp    (rank 0 of a 1-GPU run) the same window from the same state at
             k = W-2 in the other precision batched and in plain FP64 (one
             replica at a time), two untimed iterations then K timed."""
    import numpy as np
    import torch

    import scft_string_b200 as S
    from scft_string_b200 import dist as D
    from scft_string_b200.configs import fields

    torch.cuda.set_device(dev)
    if world > 1:
        D.init("nccl", device=torch.device("cuda", dev))

    def barrier():
        D.barrier(world)
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return D.max_over_ranks(v, world, device="cuda")

    wm, wp = fields(cfg)
    strn = cfg["strn"]
    ctx = S.StringSolver(cfg, precision=a.precision, batched=not a.plain, device=dev)
    for ii in range(strn):
        ctx.set_fields(ii, wm[ii], wp[ii])
    groups, wide, persist, tune_ms = ctx.autotune()  # slot groups, pencil tiles, launches per step
    ctx.solve_field0_all(5000, 1e-4)           # prelude, scft.cu:1105
    nsterp = 4000                              # scft.cu:1102
    M = ctx.M
    W0 = max(2, a.warmup)
    pinned = lambda: torch.empty((strn, 2 * M), dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    host_w2, host_w = pinned(), pinned()
    ctx.string_begin(nsterp, 1e-3)
    for k in range(W0):
        if k == W0 - 2:
            for ii in range(strn):
                ctx.get_fields(ii, out=host_w2[ii])
        ctx.string_step()
    for ii in range(strn):
        ctx.get_fields(ii, out=host_w[ii])     # the state at k = W
    # ---- value: K iterations with device-resident fields
    barrier()
    clk = Clocks(dev) if rank == 0 else None
    ctx.reset_stats()
    ctx.timer_mark(0)
    reps = [ctx.string_step() for _ in range(a.steps)]
    ctx.timer_mark(1)
    ms = ctx.timer_elapsed_ms(0, 1)
    barrier()
    clocks = clk.stop() if clk else None
    st = ctx.stats()
    ms_max = max_over_ranks(ms)
    # ---- e2e: the same iterations from the host copy at k = W; H2D + step + D2H every iteration
    host = pinned()
    host[:] = host_w
    ctx.string_end()
    ctx.string_resume(W0, nsterp, 1e-3)
    barrier()
    ctx.timer_mark(2)
    reps_e2e = []
    for _ in range(a.steps):
        for ii in range(strn):
            ctx.set_fields_2m(ii, host[ii])      # H2D from pinned host memory
        reps_e2e.append(ctx.string_step())
        for ii in range(strn):
            ctx.get_fields(ii, out=host[ii])     # D2H into pinned host memory
    ctx.timer_mark(3)
    e2e_ms = max_over_ranks(ctx.timer_elapsed_ms(2, 3))
    barrier()
    same = all(x["errtot"] == y["errtot"] for x, y in zip(reps, reps_e2e))
    out = dict(ms=ms_max, reps=reps, stats=st, clocks=clocks, e2e_ms=e2e_ms, ctx=ctx, M=M, W0=W0,
               e2e_same_iterations=same,
               schedule={"slot_groups": groups, "wide_pencil_tiles": bool(wide),
                         "persistent_step_launch": bool(persist),
                         "props_round_ms": {f"g{1 << (c % 3)}_tile{1 + (c // 3) % 2}_{'persistent' if c >= 6 else 'four'}":
                                            v for c, v in enumerate(tune_ms) if v > 0}})
    # ---- the other precision (batched) and plain FP64 on the same window
    if rank == 0 and world == 1 and not a.no_fp64:
        other = "fp64" if a.precision == "fp32" else "fp32"
        legs = [(f"{other}_batched", other, True)]
        if not (a.precision == "fp64" and a.plain):
            legs.append(("fp64_plain", "fp64", False))
        res = {}
        for name, prec, batched in legs:
            c = S.StringSolver(cfg, precision=prec, batched=batched, device=dev)
            for ii in range(strn):
                c.set_fields_2m(ii, host_w2[ii])
            if batched:
                c.autotune()
            c.string_resume(W0 - 2, nsterp, 1e-3)
            c.string_step()
            c.string_step()  # untimed: graph capture of the iteration's props rounds
            c.reset_stats()
            c.timer_mark(0)
            rr = [c.string_step() for _ in range(a.steps)]
            c.timer_mark(1)
            t = c.timer_elapsed_ms(0, 1)
            s2 = c.stats()
            res[name] = dict(iters_per_s=a.steps / (t / 1e3),
                             contour_steps_per_s=s2["contour_steps"] / s2["props_seconds"],
                             props_per_replica_iter=s2["props_calls"] / (a.steps * strn),
                             iters=a.steps, window=f"k={W0}..{W0 + a.steps - 1}",
                             errtot_last=rr[-1]["errtot"])
            c.close()
        out["cmp"] = res
        # FP32 propagator against FP64 at identical fields: the state at k = W
        one64 = S.StringSolver(dict(cfg, strn=1), precision="fp64", device=dev)
        one32 = S.StringSolver(dict(cfg, strn=1), precision="fp32", device=dev)
        dF, dq, dr = [], [], []
        for ii in range(strn):
            w = np.ascontiguousarray(host_w[ii])
            F64, q64, r64 = f_per_chain(one64, cfg, w)
            F32, q32, r32 = f_per_chain(one32, cfg, w)
            dF.append(abs(F32 - F64))
            dq.append(abs(q32 - q64) / max(1e-300, abs(q64)))
            dr.append(float(np.abs(r32 - r64).max()))
        one64.close()
        one32.close()
        out["fp32_err"] = {"at": f"fields of every replica at k={W0}",
                           "F_per_chain": dF, "lnQ_rel": dq, "rhoA_maxabs": dr}
    D.finalize(world)
    return out


def main():
    a = parse()
    rank, world, dev = dist_env()
    from scft_string_b200.configs import STRING_64
    cfg = dict(STRING_64)
    if a.profile_round > 0:
        return profile_round(a, cfg)
    if a.workload == "uneven24":
        return run_uneven(a) if rank == 0 else 0
    if a.workload == "mixed128":
        return run_mixed128(a) if rank == 0 else 0
    if a.workload == "adjoint96":
        return run_adjoint96(a) if rank == 0 else 0
    if a.workload == "tolerance":
        return run_tolerance(a) if rank == 0 else 0
    if a.impl == "reference":
        if rank != 0:
            return 0
        from oracle.refrun import time_iterations
        # the same window as our arm: iterations k = W..W+K-1 after the prelude
        r = time_iterations(cfg, max(2, a.warmup), a.steps)
        if "unavailable" in r:
            print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
            return 0
        v = r["iters_per_s"]
        line = {"metric": METRIC, "value": v, "unit": "string iters/s", "n_gpus": 1,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / v,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded fields, scft_string_b200.configs)",
                "config": {"workload": cfg["name"], "replicas": cfg["strn"], "grid": list(cfg["m"]),
                           "N": cfg["N"], "ens": cfg["ens"],
                           "window": f"iterations k={max(2, a.warmup)}..{max(2, a.warmup) + a.steps - 1} "
                                     "after the W+ prelude",
                           "program": "reference scft.cu built for sm_100a (oracle/build_ref.sh), "
                                      "single rank owning every replica"},
                "impl": "reference",
                "reference_run": {"device": "B200 GPU: the reference's only implementation is CUDA "
                                            "with cuFFT (it has no CPU path)",
                                  "host_threads": 1, "timing": "host timestamps printed at the start "
                                  "of each iteration (KSTART), iterations W..W+K-1",
                                  "props_calls_seen": r["props_lines"]},
                "e2e": {"value": v, "unit": "string iters/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        if not a.no_cpu and r.get("props_in_window"):
            line["cpu_baseline"] = cpu_baseline(cfg, r["props_in_window"] / (a.steps * cfg["strn"]))
        print(json.dumps(line))
        return 0

    r = run_ours(a, cfg, rank, world, dev)
    if rank != 0:
        return 0
    st, reps = r["stats"], r["reps"]
    M = r["M"]
    b = 4 if a.precision == "fp32" else 8
    step_bytes = 8 * M * b                              # algorithmic bytes per replica contour step
    achieved = step_bytes * st["contour_steps"] / st["props_seconds"] / 1e9
    peak, peak_kind = peaks()
    traffic = profiled_traffic(a.precision)
    from scft_string_b200 import dist as D
    value = D.job_rate(a.steps, world, r["ms"])
    props_per_iter = st["props_calls"] / (a.steps * cfg["strn"])
    import math
    flops = 30.0 * M * math.log2(M) * st["contour_steps"] / st["props_seconds"] / 1e12
    W0 = r["W0"]
    window = f"iterations k={W0}..{W0 + a.steps - 1} after the W+ prelude"
    line = {
        "metric": METRIC, "value": value, "unit": "string iters/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["ms"] / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if a.precision == "fp32" else "f64",
        "data": "synthetic (seeded fields, scft_string_b200.configs)",
        "config": {"workload": cfg["name"], "replicas": cfg["strn"], "grid": list(cfg["m"]),
                   "N": cfg["N"], "ens": cfg["ens"], "precision": a.precision,
                   "batched": not a.plain, "parallelism": f"replicas-only x{world}",
                   "schedule": r["schedule"], "window": window,
                   "l2": "inputs larger than L2 (propagator store "
                         f"{cfg['strn'] * (cfg['N'] + 1) * 2 * M * b / 1e9:.1f} GB per props round)"},
        "errtot_last": reps[-1]["errtot"], "props_per_replica_iter": props_per_iter,
        "contour_steps_per_s": st["contour_steps"] / st["props_seconds"],
        "gpu_launches": st["kernel_launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic,
                     "unit_of_work": "replica contour step (q and q^dagger advanced by ds)",
                     "algorithmic_bytes_per_unit": step_bytes,
                     "fp32_tflops" if b == 4 else "fp64_tflops": flops,
                     "alu": {"achieved": flops, "peak": alu_peak_tflops(a.precision), "unit": "TFLOP/s",
                             "frac": flops / alu_peak_tflops(a.precision), "peak_kind": "nominal",
                             "flops_per_unit": 30 * M * math.log2(M),
                             "note": "30 M log2 M algorithmic FFT flops per replica contour step against "
                                     "SMs x FMA lanes x 2 x max SM clock of the path's precision"},
                     "max_frac": max(achieved / peak, flops / alu_peak_tflops(a.precision))},
        "e2e": {"value": world * a.steps / (r["e2e_ms"] / 1e3), "unit": "string iters/s",
                "h2d_bytes_per_step": cfg["strn"] * 2 * M * 8,
                "d2h_bytes_per_step": cfg["strn"] * 2 * M * 8,
                "window": window + " (the same iterations as value, continued from a host copy of the "
                          "fields at their start)",
                "same_iterations_as_value": r["e2e_same_iterations"]},
        "clocks": r["clocks"],
    }
    if "cmp" in r:
        c = r["cmp"]
        line["same_window_cmp"] = c
        if a.precision == "fp32" and "fp64_plain" in c:
            line["speedup_vs_fp64_plain"] = value / c["fp64_plain"]["iters_per_s"]
        if "fp64_plain" in c and "fp32_batched" in c:
            line["fp32_batched_vs_fp64_plain"] = c["fp32_batched"]["iters_per_s"] / c["fp64_plain"]["iters_per_s"]
        if a.precision == "fp64" and not a.plain and "fp64_plain" in c:
            line["fp64_batched_vs_fp64_plain"] = value / c["fp64_plain"]["iters_per_s"]
    if "fp32_err" in r:
        line["fp32_vs_fp64_at_identical_fields"] = r["fp32_err"]
    if world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(cfg, props_per_iter)
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
