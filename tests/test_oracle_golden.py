"""Pins the FP64 oracle to the reference program run on a B200: the
reference's own trace (per-iteration errs/errs3 of solve_field, FreeE values,
number of props calls) for each seeded case of tests/golden/cases.py."""
import numpy as np
import pytest

import oracle as O
from cases import CASES
from replay import initial_fields, load_fixture, ref_trace


def run_oracle(c):
    wm, wp, springsteps = initial_fields(c)
    s = O.Solver(c["m"], c["D"], c["N"], c["alpha"], c["ens"], c["phidb"], c["chi"], c["f"],
                 c["strn"], c["fix"], c["dostring"], springsteps=springsteps)
    for ii in range(c["strn"]):
        s.set_fields(ii, wm[ii], wp[ii])
    for ii in range(c["strn"]):
        s.solve_field0(ii, 5000, 1e-4)
    k, recs, errs, errs3 = s.solve_field(c["nsterp"])
    fe = s.free_energy()
    return s, k, errs, errs3, fe


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_trace(name):
    fx = load_fixture(name)
    ref = ref_trace(fx)
    c = fx["params"]
    s, k, errs, errs3, fe = run_oracle(c)
    assert k == c["nsterp"] == len(ref["errs"])
    assert s.props_calls() == ref["nprops"]
    tol = 1e-10
    assert np.allclose(errs, ref["errs"], rtol=tol, atol=1e-300)
    assert np.allclose(errs3, ref["errs3"], rtol=tol, atol=1e-300)
    last = ref["final_freee"]
    assert np.allclose(fe["FEs0"], last[:, 1], rtol=tol)
    assert np.allclose(fe["FEs1"], last[:, 2], rtol=tol, atol=1e-12)
    assert np.allclose(fe["phctot"], last[:, 3], rtol=tol)
    # the win files the reference wrote at the end (%.6lf); replicas with
    # doiis == 0 (fixed ends) were last written after the prelude (scft.cu:1141)
    doiis = s.doiis()
    for ii in range(c["strn"]):
        txt = fx["files"].get(f"win{ii}")
        if txt is None or doiis[ii] != 1:
            continue
        vals = np.array(txt.split(), float).reshape(-1, 2)
        W = s.W(ii)
        assert np.abs(vals[:, 0] - W[: s.M]).max() <= 5.1e-7
        assert np.abs(vals[:, 1] - W[s.M: 2 * s.M]).max() <= 5.1e-7
