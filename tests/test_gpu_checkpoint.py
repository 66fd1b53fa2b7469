"""Binary FP64 checkpoint: a round trip restores box and fields bit for bit;
a corrupted or mismatched file is refused."""
import numpy as np
import pytest

import scft_string_b200 as S
from scft_string_b200.configs import STRING_64, fields

pytestmark = pytest.mark.gpu


def test_checkpoint_round_trip_and_refusals(built_lib, tmp_path):
    c = dict(STRING_64, m=(16, 16, 16), D=(2.5, 2.5, 2.5), N=20, strn=3)
    wm, wp = fields(c)
    a = S.StringSolver(c)
    for ii in range(3):
        a.set_fields(ii, wm[ii], wp[ii] + 0.1 * ii)
    a.set_box([2.4, 2.6, 2.5])
    path = str(tmp_path / "f.ckpt")
    a.save_checkpoint(path)
    b = S.StringSolver(c, precision="fp32")
    b.load_checkpoint(path)
    np.testing.assert_array_equal(b.get_box(), [2.4, 2.6, 2.5])
    for ii in range(3):
        np.testing.assert_array_equal(b.get_fields(ii), a.get_fields(ii))
    raw = bytearray(open(path, "rb").read())
    raw[-100] ^= 0x01                      # flip one bit of the last replica's fields
    bad = str(tmp_path / "bad.ckpt")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(S.ScftError):
        b.load_checkpoint(bad)
    other = S.StringSolver(dict(c, strn=2))
    with pytest.raises(S.ScftError):
        other.load_checkpoint(path)
