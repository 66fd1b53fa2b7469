"""The plain FP64 GPU path replays the reference program's own runs (golden
traces recorded on a B200) with the reference's main() sequence; errors per
iteration, props-call counts and free energies agree to 1e-10 relative."""
import numpy as np
import pytest

import scft_string_b200 as S
from cases import CASES
from replay import initial_fields, load_fixture, ref_trace

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run_gpu(c, batched=True, precision="fp64"):
    wm, wp, springsteps = initial_fields(c)
    ctx = S.StringSolver(c, precision=precision, batched=batched, springsteps=springsteps)
    for ii in range(c["strn"]):
        ctx.set_fields(ii, wm[ii], wp[ii])
    ctx.solve_field0_all(c.get("prelude", 5000), 1e-4)
    k, recs, errs, errs3 = ctx.solve_field(c["nsterp"])
    fe = ctx.free_energy()
    return ctx, k, recs, errs, errs3, fe


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference_trace(built_lib, name, batched):
    fx = load_fixture(name)
    ref = ref_trace(fx)
    c = fx["params"]
    ctx, k, recs, errs, errs3, fe = run_gpu(c, batched=batched)
    assert k == len(ref["errs"])
    assert ctx.stats()["props_calls"] == ref["nprops"]
    assert np.allclose(errs, ref["errs"], rtol=TOL, atol=1e-300)
    assert np.allclose(errs3, ref["errs3"], rtol=TOL, atol=1e-300)
    last = ref["final_freee"]
    assert np.allclose(fe["FEs0"], last[:, 1], rtol=TOL)
    assert np.allclose(fe["FEs1"], last[:, 2], rtol=TOL, atol=1e-12)
    assert np.allclose(fe["phctot"], last[:, 3], rtol=TOL)
    # -lnQ of the final props of every replica
    for ii in range(c["strn"]):
        _, lnQ, _ = ctx.get_conc(ii)
        assert abs(-lnQ - last[ii, 1]) <= TOL * max(1.0, abs(last[ii, 1]))


def test_fp64_plain32_c1_trace(built_lib):
    """The 32^3, N=100 single-replica canonical workload: prelude, 200
    iterations and final FreeE against the reference's PROPS trace."""
    fx = load_fixture("plain32_c1")
    ref = ref_trace(fx)
    c = fx["params"]
    ctx, k, recs, errs, errs3, fe = run_gpu(c, batched=True)
    assert k == 200
    assert ctx.stats()["props_calls"] == ref["nprops"]
    assert np.allclose(errs, ref["errs"], rtol=TOL)
    last = ref["final_freee"]
    F = last[:, 1] + last[:, 2]
    assert np.allclose(fe["FEs"], F, rtol=TOL)
    _, lnQ, phis = ctx.get_conc(0)
    assert abs(lnQ - ref["props"][-1, 2]) <= TOL * abs(ref["props"][-1, 2])
    assert np.allclose(phis, ref["props"][-1, 3:8], rtol=TOL)


@pytest.mark.parametrize("name", ["string64_c2", "adjoint96_c4"])
def test_fp64_benchmark_configs_match_reference_trace(built_lib, name):
    """The benchmarked 16-replica 64^3 string (W+ prelude, five string
    iterations, FreeE at k = 0 and k = 4) and the 64x64x96, N = 160
    workload from its hexagonal start (20 prelude props, two iterations):
    the number of props calls, the per-iteration errs/errs3, the final FreeE
    and the last props call's lnQ and phis against the reference program's
    own run."""
    try:
        fx = load_fixture(name)
    except FileNotFoundError:
        pytest.skip(f"fixture ref_{name} not recorded")
    ref = ref_trace(fx)
    c = fx["params"]
    ctx, k, recs, errs, errs3, fe = run_gpu(c, batched=True)
    assert k == len(ref["errs"])
    assert ctx.stats()["props_calls"] == ref["nprops"]
    assert np.allclose(errs, ref["errs"], rtol=TOL, atol=1e-300)
    assert np.allclose(errs3, ref["errs3"], rtol=TOL, atol=1e-300)
    last = ref["final_freee"]
    assert np.allclose(fe["FEs0"], last[:, 1], rtol=TOL)
    assert np.allclose(fe["FEs1"], last[:, 2], rtol=TOL, atol=1e-12)
    assert np.allclose(fe["phctot"], last[:, 3], rtol=TOL)
    for ii in range(c["strn"]):
        _, lnQ, phis = ctx.get_conc(ii)
        assert abs(-lnQ - last[ii, 1]) <= TOL * max(1.0, abs(last[ii, 1]))
    assert abs(lnQ - ref["props"][-1, 2]) <= TOL * max(1.0, abs(ref["props"][-1, 2]))
    assert np.allclose(phis, ref["props"][-1, 3:8], rtol=TOL, atol=1e-14)
