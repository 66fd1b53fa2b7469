"""The binary checkpoint format, read on the CPU (scft_checkpoint_info runs the
load path's checks without a context or a device).  Files are written here
byte by byte from the layout: magic, u32 version, u32 problem-record size,
the record, i32 strn, i64 M, the fields, the per-replica boxes (version 2)
and the FNV-1a hash of field and box bytes.  The record only grows at its
end, so shorter (older) and longer records read too."""
import ctypes as C
import struct

import numpy as np
import pytest

import scft_string_b200 as S

M3, D3, STRN = (4, 6, 8), (2.5, 3.0, 3.5), 3


def fnv1a(data: bytes, h=1469598103934665603):
    for b in data:
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def problem_bytes(psz):
    p = S.Problem()
    for i in range(3):
        p.m[i], p.D[i] = M3[i], D3[i]
    p.N, p.strn = 20, STRN
    raw = bytes(C.string_at(C.addressof(p), C.sizeof(p)))
    return raw[:psz] if psz <= len(raw) else raw + b"\x07" * (psz - len(raw))


def write(path, version=2, psz=None, magic=b"SCFTCKP1", M=None, cut=0, flip=None):
    psz = C.sizeof(S.Problem) if psz is None else psz
    M = int(np.prod(M3)) if M is None else M
    rng = np.random.default_rng(1)
    fields = rng.normal(size=2 * int(np.prod(M3)) * STRN).tobytes()
    boxes = np.array([D3] * STRN, dtype=np.float64).tobytes() if version == 2 else b""
    h = fnv1a(fields + boxes)
    raw = bytearray(magic + struct.pack("<II", version, psz) + problem_bytes(psz) + struct.pack("<iq", STRN, M)
                    + fields + boxes + struct.pack("<Q", h))
    if flip is not None:
        raw[flip] ^= 0x01
    if cut:
        raw = raw[:-cut]
    open(path, "wb").write(bytes(raw))
    return str(path)


def test_current_layout(built_lib, tmp_path):
    info = S.checkpoint_info(write(tmp_path / "a.ckpt"))
    assert info == {"version": 2, "strn": STRN, "m": M3, "D": D3}


@pytest.mark.parametrize("version", [1, 2])
def test_older_shorter_problem_record(built_lib, tmp_path, version):
    """Records written before fields were appended (version 1 predates the
    per-replica boxes and the last two problem fields)."""
    short = C.sizeof(S.Problem) - 8
    info = S.checkpoint_info(write(tmp_path / "a.ckpt", version=version, psz=short))
    assert info == {"version": version, "strn": STRN, "m": M3, "D": D3}


def test_longer_problem_record(built_lib, tmp_path):
    info = S.checkpoint_info(write(tmp_path / "a.ckpt", psz=C.sizeof(S.Problem) + 24))
    assert info["m"] == M3 and info["strn"] == STRN


@pytest.mark.parametrize("kw", [
    dict(magic=b"SCFTCKP0"),                 # not a checkpoint
    dict(version=3),                         # unknown version
    dict(psz=16),                            # record does not reach D
    dict(psz=1 << 20),                       # implausible record size
    dict(M=7),                               # M disagrees with m
    dict(cut=1),                             # truncated hash
    dict(cut=200),                           # truncated boxes / fields
    dict(flip=-20),                          # one bit of the last box
    dict(flip=-500),                         # one bit of the fields
])
def test_refused(built_lib, tmp_path, kw):
    with pytest.raises(S.ScftError):
        S.checkpoint_info(write(tmp_path / "a.ckpt", **kw))


def test_missing_file(built_lib, tmp_path):
    with pytest.raises(S.ScftError):
        S.checkpoint_info(str(tmp_path / "none.ckpt"))
