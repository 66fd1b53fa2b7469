"""Replays a golden case (reference run recorded by tests/golden/make_ref_golden.py)
through a solver with the reference's main() sequence (scft.cu:1057-1132):
read win files (a missing file copies the previous replica and adds a spring
step, scft.cu:1065-1078), W+ prelude solve_field0(5000, 1e-4) per replica,
solve_field(nsterp), final FreeE."""
from __future__ import annotations

import gzip
import json
import os

import numpy as np

from scft_string_b200.configs import fields, hex_fields

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    with gzip.open(os.path.join(GOLDEN, f"ref_{name}.json.gz"), "rt") as fh:
        return json.load(fh)


def initial_fields(c):
    """(W- rows, W+ rows, springsteps) after the reference's win-file read."""
    wm, wp = hex_fields(c) if c.get("start") == "hex" else fields(c)
    wm, wp = wm.copy(), wp.copy()
    missing = set(c.get("missing", ()))
    springsteps, cpto0 = 0, False
    for ii in range(c["strn"]):
        if ii in missing:
            springsteps += 1
            if ii != 0:
                wm[ii], wp[ii] = wm[ii - 1], wp[ii - 1]
            else:
                cpto0 = True
    if cpto0:
        wm[0], wp[0] = wm[1], wp[1]
    return wm, wp, springsteps


def ref_trace(fx):
    strn = fx["params"]["strn"]
    e = np.array([row[1:] for row in fx["errs"]]) if fx["errs"] else np.zeros((0, 2 * strn))
    fr = np.array(fx["freee"])
    return dict(errs=e[:, 0::2], errs3=e[:, 1::2], props=np.array(fx["props"]),
                freee=fr, final_freee=fr[-strn:], nprops=len(fx["props"]))
