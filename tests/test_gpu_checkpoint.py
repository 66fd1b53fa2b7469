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


def test_older_layout_loads(built_lib, tmp_path):
    """A version 1 file with the shorter problem record of its time (no
    per-replica boxes, the record 8 bytes shorter) loads into a current
    context: the same fields, the record's box for every replica."""
    import struct
    c = dict(STRING_64, m=(16, 16, 16), D=(2.5, 2.5, 2.5), N=20, strn=2)
    wm, wp = fields(c)
    a = S.StringSolver(c)
    for ii in range(2):
        a.set_fields(ii, wm[ii], wp[ii])
    a.set_box([2.4, 2.6, 2.5])
    path = str(tmp_path / "new.ckpt")
    a.save_checkpoint(path)
    raw = open(path, "rb").read()
    psz = struct.unpack_from("<I", raw, 12)[0]
    rec = raw[16:16 + psz - 8]
    rest = raw[16 + psz:]
    M = a.M
    flds = rest[12:12 + 2 * 2 * M * 8]

    def fnv1a(data, h=1469598103934665603):
        for b in data:
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return h

    old = (b"SCFTCKP1" + struct.pack("<II", 1, psz - 8) + rec + rest[:12] + flds
           + struct.pack("<Q", fnv1a(flds)))
    opath = str(tmp_path / "old.ckpt")
    open(opath, "wb").write(old)
    assert S.checkpoint_info(opath)["version"] == 1
    b = S.StringSolver(c)
    b.set_box([3.0, 3.0, 3.0])
    b.load_checkpoint(opath)
    for ii in range(2):
        np.testing.assert_array_equal(b.get_fields(ii), a.get_fields(ii))
        np.testing.assert_array_equal(b.get_box(ii), [2.4, 2.6, 2.5])
