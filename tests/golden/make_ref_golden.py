#!/usr/bin/env python3
"""Generates the golden fixtures ``tests/golden/ref_<case>.json.gz`` by running
the reference CUDA program (built from the reference sources by
``oracle/build_ref.sh``) on the seeded cases of ``cases.py``.

Two phases, because the reference sources live only in the development
container while the reference program needs a GPU:

  python tests/golden/make_ref_golden.py --build          # here: nvcc the binaries
  python tests/golden/make_ref_golden.py --run --out DIR  # on a B200: run, write fixtures

Each fixture holds the full-precision trace the patched reference prints
(``PROPS`` per props call, ``ERRS`` per string iteration, ``FREEE`` per free
energy evaluation) and the text of every file it writes (``FEs``, ``check``,
``win<ii>``, ``rhoA_<ii>.vtk``, ``rhocB_<ii>.vtk``).
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES  # noqa: E402
from scft_string_b200.configs import (ADJOINT_96, PLAIN_32, STRING_64, fields, hex_fields, input_dat,  # noqa: E402
                                      win_text)

PRELUDE = 5000


def all_cases():
    out = dict(CASES)
    c1 = dict(PLAIN_32)
    c1["nsterp"] = 200
    c1["trace_only"] = True
    out["plain32_c1"] = c1
    # the benchmarked string: 16 replicas of 64^3, N = 128; W+ prelude and the
    # first five string iterations (FreeE at k = 0 and at the last one)
    c2 = dict(STRING_64)
    c2["nsterp"] = 5
    c2["trace_only"] = True
    out["string64_c2"] = c2
    # the 64x64x96, N = 160 adjoint workload from its hexagonal start: a short
    # W+ prelude (20 props) and two iterations of the plain method
    c4 = dict(ADJOINT_96)
    c4.update(nsterp=2, prelude=20, trace_only=True, start="hex")
    out["adjoint96_c4"] = c4
    return out


def case_fields(c):
    return hex_fields(c) if c.get("start") == "hex" else fields(c)


def binary(c):
    return os.path.join(ROOT, "oracle", "_ref",
                        f"scft_ref_s{c['strn']}_n{c['nsterp']}_p{c.get('prelude', PRELUDE)}")


def build():
    for name, c in all_cases().items():
        if not os.path.exists(binary(c)):
            subprocess.run([os.path.join(ROOT, "oracle", "build_ref.sh"), str(c["strn"]),
                            str(c["nsterp"]), str(c.get("prelude", PRELUDE))], check=True)
        print(name, binary(c))


def parse_trace(text):
    props, errs, freee = [], [], []
    for line in text.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "PROPS":
            props.append([float(v) for v in t[1:]])
        elif t[0] == "ERRS":
            errs.append([int(t[1])] + [float(v) for v in t[2:]])
        elif t[0] == "FREEE":
            freee.append([int(t[1])] + [float(v) for v in t[2:]])
    return props, errs, freee


def run_case(name, c, outdir):
    wm, wp = case_fields(c)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input.dat"), "w") as fh:
            fh.write(input_dat(c))
        for ii in range(c["strn"]):
            if ii in c.get("missing", ()):
                continue
            with open(os.path.join(d, f"win{ii}"), "w") as fh:
                fh.write(win_text(wm[ii], wp[ii]))
        p = subprocess.run([binary(c)], cwd=d, capture_output=True, text=True, timeout=3000)
        props, errs, freee = parse_trace(p.stdout)
        files = {}
        if not c.get("trace_only"):
            for fn in sorted(os.listdir(d)):
                if fn == "input.dat":
                    continue
                with open(os.path.join(d, fn)) as fh:
                    files[fn] = fh.read()
        fix = dict(case=name, params=c, returncode=p.returncode, props=props, errs=errs,
                   freee=freee, files=files, stdout_tail=p.stdout[-4000:],
                   stderr_tail=p.stderr[-2000:])
    path = os.path.join(outdir, f"ref_{name}.json.gz")
    with gzip.open(path, "wt") as fh:
        json.dump(fix, fh)
    print(name, "rc", p.returncode, "props", len(props), "iters", len(errs), "->", path, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--build", action="store_true")
    ap.add_argument("--run", action="store_true")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if a.build:
        build()
    if a.run:
        os.makedirs(a.out, exist_ok=True)
        for name, c in all_cases().items():
            if a.only and name not in a.only.split(","):
                continue
            run_case(name, c, a.out)


if __name__ == "__main__":
    main()
