"""The FP32 propagator path against the FP64 path.

Accuracy is measured at identical fields: the FP64 solver is run to a state,
the same W-, W+ go into an FP32 context, and one props of each gives
lnQ, rhoA and the free energy per chain F = -lnQ + <chi phiA phiB - wA phiA - wB phiB>
(scft.cu:820-829).  FP32 storage and transforms have an error floor that grows
with the dynamic range of q across the box (strong fields): on these small
cases the same propagator written with numpy float32 FFTs errs by 1e-5..4e-5
kT per chain, so the bound here is 1e-4 kT per chain and 1e-5 on rhoA.
Trajectories (which pass through the reference's error-tolerance stops) are
compared more loosely."""
import numpy as np
import pytest

import scft_string_b200 as S
from cases import CASES
from replay import initial_fields

pytestmark = pytest.mark.gpu


def solve(c, precision, iters):
    wm, wp, springsteps = initial_fields(c)
    ctx = S.StringSolver(c, precision=precision, batched=True, springsteps=springsteps)
    for ii in range(c["strn"]):
        ctx.set_fields(ii, wm[ii], wp[ii])
    ctx.solve_field0_all(5000, 1e-4)
    k, recs, errs, errs3 = ctx.solve_field(iters)
    return ctx, recs


def f_at_fields(ctx, c, W):
    """props of every replica at fields W (strn x 2M): F per chain, rhoA, lnQ."""
    M = ctx.M
    F, rho, lnq = [], [], []
    for ii in range(c["strn"]):
        ctx.set_fields_2m(ii, np.ascontiguousarray(W[ii]))
        ctx.props(ii)
        conc, lnQ, _ = ctx.get_conc(ii)
        pA, pB = conc[:M], conc[M:2 * M]
        wa, wb = W[ii][:M] + W[ii][M:], W[ii][M:] - W[ii][:M]
        F.append(-lnQ + np.mean(c["chi"] * pA * pB - wa * pA - wb * pB))
        rho.append(pA)
        lnq.append(lnQ)
    return np.array(F), np.array(rho), np.array(lnq)


@pytest.mark.parametrize("name", ["string_mixed", "string_c", "plain_c"])
def test_fp32_free_energy_at_same_fields(built_lib, name):
    c = dict(CASES[name])
    ctx64, _ = solve(c, "fp64", 6)
    W = np.stack([ctx64.get_fields(ii) for ii in range(c["strn"])])
    ctx32 = S.StringSolver(c, precision="fp32", batched=True)
    F64, r64, q64 = f_at_fields(ctx64, c, W)
    F32, r32, q32 = f_at_fields(ctx32, c, W)
    print(name, "dF", np.abs(F32 - F64).max(), "drhoA", np.abs(r32 - r64).max())
    assert np.abs(F32 - F64).max() <= 1e-4
    assert np.abs(r32 - r64).max() <= 1e-5


def test_fp32_free_energy_64cubed_string(built_lib):
    """Four replicas of the 64^3, N=128 string workload after the prelude
    and 2 string iterations in FP64 (the lamellar end has the largest
    dynamic range; numpy float32 at the unrelaxed fields errs by 4e-3 in F)."""
    from scft_string_b200.configs import STRING_64
    c = dict(STRING_64)
    c["strn"] = 4
    ctx64, _ = solve(c, "fp64", 2)
    W = np.stack([ctx64.get_fields(ii) for ii in range(c["strn"])])
    ctx32 = S.StringSolver(c, precision="fp32", batched=True)
    F64, r64, _ = f_at_fields(ctx64, c, W)
    F32, r32, _ = f_at_fields(ctx32, c, W)
    print("64^3 dF", np.abs(F32 - F64), "drhoA", np.abs(r32 - r64).max(axis=1))
    assert np.abs(F32 - F64).max() <= 1e-2
    assert np.abs(r32 - r64).max() <= 1e-3


@pytest.mark.parametrize("name", ["string_mixed", "plain_c"])
def test_fp32_trajectory_tracks_fp64(built_lib, name):
    c = dict(CASES[name])
    _, rec64 = solve(c, "fp64", 12)
    _, rec32 = solve(c, "fp32", 12)
    e64 = np.array([r["errtot"] for r in rec64])
    e32 = np.array([r["errtot"] for r in rec32])
    assert np.allclose(e32, e64, rtol=1e-2)
    FE64 = [r["FE"] for r in rec64 if r["did_freee"]]
    FE32 = [r["FE"] for r in rec32 if r["did_freee"]]
    assert np.allclose(FE32, FE64, rtol=0, atol=1e-4 * c["strn"])
