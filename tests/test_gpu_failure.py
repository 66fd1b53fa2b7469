"""Failure paths on the GPU, made to happen without a GPU fault.

* Timeout: one bounded device wait on a barrier that nothing completes (its
  bulk copy is never issued) runs out after a short poll limit, exactly as a
  wait on a lost copy in the step kernels would; the call returns
  SCFT_TIMEOUT, the error word is cleared, and the same context's next props
  equals that of a fresh context bit for bit.
* NaN: a NaN put into one replica's W- on the host makes the W+ relaxation
  return SCFT_NAN_DETECTED at the point where the reference asserts
  (scft.cu:539: assert(err == err)); once valid fields are set again the same
  context solves exactly as a fresh one does.
"""
import numpy as np
import pytest

import scft_string_b200 as S

pytestmark = pytest.mark.gpu

TIMEOUT = 4
NAN_DETECTED = 2


def _ctx(m, prec, strn=1):
    D = (4.0, 4.0, 4.0)
    return S.Context(m, D, 24, chi=12.0, f=0.45, phidb=0.8, ens=2, strn=strn, dostring=0 if strn == 1 else 1,
                     precision=prec)


def _fields(m, seed=5):
    rng = np.random.default_rng(seed)
    M = int(np.prod(m))
    return rng.normal(0, 1.5, M), rng.normal(0, 0.3, M)


@pytest.mark.parametrize("m,prec", [((32, 32, 32), "fp32"), ((32, 32, 32), "fp64"), ((16, 12, 10), "fp64")])
def test_bounded_wait_times_out_and_context_survives(built_lib, m, prec):
    wm, wp = _fields(m)
    ctx = _ctx(m, prec)
    ctx.set_fields(0, wm, wp)
    assert ctx.selftest_timeout(1000) == TIMEOUT
    assert "gave up" in S.lib().scft_last_error(ctx.h).decode()
    # the error word was cleared: a second self-test times out again (not a stale code)
    assert ctx.selftest_timeout(10) == TIMEOUT
    ctx.props(0)
    got, lnq, phis = ctx.get_conc(0)
    fresh = _ctx(m, prec)
    fresh.set_fields(0, wm, wp)
    fresh.props(0)
    ref, lnq0, phis0 = fresh.get_conc(0)
    assert lnq == lnq0
    assert np.array_equal(got, ref)
    assert np.array_equal(phis, phis0)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_nan_in_field_is_reported_and_context_recovers(built_lib, prec):
    m = (16, 12, 10)
    M = int(np.prod(m))
    ctx = _ctx(m, prec, strn=3)
    good = [_fields(m, seed) for seed in (1, 2, 3)]
    for ii, (wm, wp) in enumerate(good):
        ctx.set_fields(ii, wm, wp)
    bad = good[1][0].copy()
    bad[M // 3] = np.nan
    ctx.set_fields(1, bad, good[1][1])
    with pytest.raises(S.ScftError) as ei:
        ctx.solve_field0(1, 100, 1e-4)
    assert ei.value.status == NAN_DETECTED
    with pytest.raises(S.ScftError) as ei:
        ctx.solve_field0_all(100, 1e-4)
    assert ei.value.status == NAN_DETECTED
    # valid fields again: the same context solves as a fresh one does
    for ii, (wm, wp) in enumerate(good):
        ctx.set_fields(ii, wm, wp)
    k = ctx.solve_field0_all(200, 1e-4)
    fresh = _ctx(m, prec, strn=3)
    for ii, (wm, wp) in enumerate(good):
        fresh.set_fields(ii, wm, wp)
    k0 = fresh.solve_field0_all(200, 1e-4)
    assert list(k) == list(k0)
    for ii in range(3):
        assert np.array_equal(ctx.get_fields(ii), fresh.get_fields(ii))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_string_resume_continues_the_run(built_lib, prec):
    """A run stopped at iteration k0 and continued from its fields with
    scft_string_resume gives the same iterations, FreeE at k = 50 included,
    as the uninterrupted run: what a restart from a checkpoint relies on."""
    from cases import CASES

    from scft_string_b200.configs import fields
    c = dict(CASES["string_mixed"])
    wm, wp = fields(c)

    def fresh():
        ctx = S.StringSolver(c, precision=prec)
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        ctx.solve_field0_all(5000, 1e-4)
        return ctx

    a = fresh()
    a.string_begin(4000)
    full = [a.string_step() for _ in range(53)]
    b = fresh()
    b.string_begin(4000)
    for _ in range(47):
        b.string_step()
    W = [np.ascontiguousarray(b.get_fields(ii)) for ii in range(c["strn"])]
    r = S.StringSolver(c, precision=prec)
    for ii in range(c["strn"]):
        r.set_fields_2m(ii, W[ii])
    r.string_resume(47, 4000)
    tail = [r.string_step() for _ in range(6)]
    for x, y in zip(full[47:], tail):
        assert x["k"] == y["k"]
        assert x["did_freee"] == y["did_freee"]
        assert x["errtot"] == y["errtot"]
        assert x["FE"] == y["FE"]
    assert tail[3]["did_freee"] == 1  # k = 50
    for ii in range(c["strn"]):
        assert np.array_equal(a.get_fields(ii), r.get_fields(ii))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_smaller_context_keeps_larger_contexts_launchable(built_lib, prec):
    """The runtime-shaped kernels serve every context: creating a context of
    a small grid (and running its adjoint) after one of a large grid must not
    lower the shared-memory limit the large one launches with."""
    big, small = (30, 28, 24), (6, 5, 9)
    wm, wp = _fields(big)
    a = S.Context(big, (4.0, 4.0, 3.5), 20, chi=12.0, f=0.45, phidb=0.8, ens=2, strn=1, dostring=0, precision=prec)
    a.set_fields(0, wm, wp)
    a.props(0)
    ref = a.get_conc(0)
    _, sref = a.stress(0)
    b = S.Context(small, (2.0, 2.0, 3.0), 20, chi=12.0, f=0.45, phidb=0.8, ens=2, strn=1, dostring=0,
                  precision=prec)
    bw, bp = _fields(small)
    b.set_fields(0, bw, bp)
    b.props(0)
    b.stress(0)
    a.props(0)
    got = a.get_conc(0)
    assert np.array_equal(got[0], ref[0]) and got[1] == ref[1]
    _, s2 = a.stress(0)
    assert np.array_equal(s2, sref)
