"""The FP32 propagator path against the FP64 path on the same string runs:
free energy per chain within 1e-6 kT, rhoA within 1e-5 (max abs), and the
same RMS residual trajectory to FP32 rounding."""
import numpy as np
import pytest

import scft_string_b200 as S
from cases import CASES
from replay import initial_fields

pytestmark = pytest.mark.gpu


def run(c, precision, iters):
    wm, wp, springsteps = initial_fields(c)
    ctx = S.StringSolver(c, precision=precision, batched=True, springsteps=springsteps)
    for ii in range(c["strn"]):
        ctx.set_fields(ii, wm[ii], wp[ii])
    ctx.solve_field0_all(5000, 1e-4)
    k, recs, errs, errs3 = ctx.solve_field(iters)
    fe = ctx.free_energy()
    rhoA = np.stack([ctx.get_conc(ii)[0][: ctx.M] for ii in range(c["strn"])])
    return fe, rhoA, recs


@pytest.mark.parametrize("name", ["string_mixed", "string_c", "plain_c"])
def test_fp32_string_matches_fp64(built_lib, name):
    c = dict(CASES[name])
    f64, r64, rec64 = run(c, "fp64", 12)
    f32, r32, rec32 = run(c, "fp32", 12)
    assert np.abs(f32["FEs"] - f64["FEs"]).max() <= 1e-6
    assert np.abs(r32 - r64).max() <= 1e-5
    e64 = np.array([r["errtot"] for r in rec64])
    e32 = np.array([r["errtot"] for r in rec32])
    assert np.allclose(e32, e64, rtol=1e-4)


def test_fp32_string_64cubed_matches_fp64(built_lib):
    """Four replicas of the 64^3, N=128 string workload, 3 iterations."""
    from scft_string_b200.configs import STRING_64
    c = dict(STRING_64)
    c["strn"] = 4
    f64, r64, _ = run(c, "fp64", 3)
    f32, r32, _ = run(c, "fp32", 3)
    assert np.abs(f32["FEs"] - f64["FEs"]).max() <= 1e-6
    assert np.abs(r32 - r64).max() <= 1e-5
