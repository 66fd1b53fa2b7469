"""The props-round autotuner (slot groups x pencil tile width) changes only
the schedule: after it has run every candidate, the densities left by the last
one (two groups, wide tensor-map tiles) equal those of a plain props call bit
for bit."""
import numpy as np
import pytest

import scft_string_b200 as S
from scft_string_b200.configs import STRING_64, fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_autotune_schedules_give_identical_densities(built_lib, precision):
    c = dict(STRING_64, m=(32, 32, 32), D=(4.0, 4.0, 4.0), N=40, strn=4)
    wm, wp = fields(c)
    ctx = S.StringSolver(c, precision=precision)
    for ii in range(c["strn"]):
        ctx.set_fields(ii, wm[ii], wp[ii])
    ref = []
    for ii in range(c["strn"]):
        ctx.props(ii)
        ref.append(ctx.get_conc(ii))
    groups, wide, persist, t = ctx.autotune()
    assert groups in (1, 2) and wide in (0, 1) and persist in (0, 1) and len(t) == 12
    # 32^3: tensor-map pencils and the persistent launch ran with 1 and 2 groups;
    # 4 groups need 16 replicas
    assert all(t[c] > 0 for c in range(12) if c % 3 != 2), t
    assert all(t[c] == -1 for c in range(12) if c % 3 == 2), t
    for ii in range(c["strn"]):
        conc, lnq, phis = ctx.get_conc(ii)
        np.testing.assert_array_equal(conc, ref[ii][0])
        assert lnq == ref[ii][1]
    print(precision, "schedule", groups, wide, "round ms", t)


def test_persistent_step_launch_matches_four_launches(built_lib, monkeypatch):
    """64^3 FP32 runs the register-resident step kernels; one persistent
    launch per contour step (work items claimed in order, waits bounded) and
    four launches per step run the same arithmetic, so the densities and lnQ
    of a props round agree bit for bit, and the autotuner's four schedules
    leave them unchanged."""
    c = dict(STRING_64, N=40, strn=4)
    wm, wp = fields(c)

    monkeypatch.setenv("SCFT_REG64", "1")

    def run(no_persist):
        if no_persist:
            monkeypatch.setenv("SCFT_NO_PERSIST", "1")
        else:
            monkeypatch.delenv("SCFT_NO_PERSIST", raising=False)
        ctx = S.StringSolver(c, precision="fp32")
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        ctx.solve_field0_all(2, 0.0)  # one batched props round of every replica (then a W+ update)
        return ctx, [ctx.get_conc(ii) for ii in range(c["strn"])]

    ctx, persistent = run(False)
    launches = ctx.stats()["kernel_launches"]
    ctx4, four = run(True)
    assert ctx4.stats()["kernel_launches"] > 3 * launches  # 4 N + 6 against N + 6 per round
    for (ca, qa, pa), (cb, qb, pb) in zip(persistent, four):
        np.testing.assert_array_equal(ca, cb)
        assert qa == qb
    ref = []
    for ii in range(c["strn"]):  # densities at the fields after the W+ update
        ctx.props(ii)
        ref.append(ctx.get_conc(ii)[0])
    groups, wide, persist, t = ctx.autotune()
    assert groups in (1, 2) and wide == 0 and persist in (0, 1)
    assert all(t[c] > 0 for c in (0, 1, 6, 7)) and all(t[c] == -1 for c in range(12) if c not in (0, 1, 6, 7)), t
    for ii in range(c["strn"]):
        conc, lnq, _ = ctx.get_conc(ii)
        np.testing.assert_array_equal(conc, ref[ii])
    print("round ms", t)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_persistent_launch_of_the_shared_memory_kernels(built_lib, monkeypatch, precision):
    """The shared-memory step kernels of the compile-time shapes as one
    persistent launch per contour step (SCFT_PERSIST=1): a props round of four
    64^3 replicas gives the densities and lnQ of four launches per step bit
    for bit, with N + 6 launches per round instead of 4 N + 6."""
    monkeypatch.delenv("SCFT_REG64", raising=False)
    c = dict(STRING_64, N=40, strn=4)
    wm, wp = fields(c)

    def run(persist):
        monkeypatch.setenv("SCFT_PERSIST", persist)
        ctx = S.StringSolver(c, precision=precision)
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        ctx.solve_field0_all(2, 0.0)
        return ctx, [ctx.get_conc(ii) for ii in range(c["strn"])]

    c1, one = run("1")
    c4, four = run("0")
    assert c4.stats()["kernel_launches"] > 3 * c1.stats()["kernel_launches"]
    for (ca, qa, pa), (cb, qb, pb) in zip(one, four):
        np.testing.assert_array_equal(ca, cb)
        assert qa == qb


@pytest.mark.parametrize("persist", ["0", "1"])
def test_four_slot_groups_match_two(built_lib, monkeypatch, persist):
    """Four slot groups (two after another on each of the two streams) change
    only the schedule: a props round of 16 replicas, and the W+ relaxation's
    partial batches that fall back to two groups, give the densities and lnQ
    of two groups bit for bit, with four launches per step and with the
    persistent launch (whose counters are per stream)."""
    monkeypatch.delenv("SCFT_REG64", raising=False)
    monkeypatch.setenv("SCFT_PERSIST", persist)
    c = dict(STRING_64, m=(32, 32, 32), D=(4.0, 4.0, 4.0), N=40, strn=16)
    wm, wp = fields(c)

    def run(groups):
        monkeypatch.setenv("SCFT_GROUPS", groups)
        ctx = S.StringSolver(c, precision="fp32")
        for ii in range(c["strn"]):
            ctx.set_fields(ii, wm[ii], wp[ii])
        k = ctx.solve_field0_all(30, 1e-4)
        return k, [ctx.get_conc(ii) for ii in range(c["strn"])], [ctx.get_fields(ii) for ii in range(c["strn"])]

    k4, conc4, w4 = run("4")
    k2, conc2, w2 = run("2")
    assert list(k4) == list(k2)
    for (ca, qa, _), (cb, qb, _) in zip(conc4, conc2):
        np.testing.assert_array_equal(ca, cb)
        assert qa == qb
    for a, b in zip(w4, w2):
        np.testing.assert_array_equal(a, b)
