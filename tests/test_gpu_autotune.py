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
    groups, wide, t = ctx.autotune()
    assert groups in (1, 2) and wide in (0, 1) and len(t) == 4
    assert all(v > 0 for v in t), t          # 32^3 has tensor-map pencils: all four schedules ran
    for ii in range(c["strn"]):
        conc, lnq, phis = ctx.get_conc(ii)
        np.testing.assert_array_equal(conc, ref[ii][0])
        assert lnq == ref[ii][1]
    print(precision, "schedule", groups, wide, "round ms", t)
