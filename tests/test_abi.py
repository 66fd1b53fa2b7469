"""The C-ABI library builds for sm_100a, loads, and exports every function
include/scft_b200.h declares; scft_create checks a problem on the host and
answers without a device (no GPU calls, no CPU fallback)."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

import scft_string_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "scft_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(scft_[A-Za-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(S.EXPORTS) == names


def test_status_strings(built_lib):
    S.lib()
    assert S.lib().scft_status_string(0) == b"ok"
    assert S.lib().scft_status_string(3) == b"bad input"


def _problem(**kw):
    p = S.Problem()
    base = dict(m=(8, 8, 8), D=(2.0, 2.0, 2.0), N=20, alpha=0.1, ens=1, phidb=0.8, chi=12.0, f=0.5, strn=2,
                precision=0, batched=1, fcont=0)
    base.update(kw)
    for k, v in base.items():
        if k in ("m", "D"):
            arr = getattr(p, k)
            for i in range(3):
                arr[i] = v[i]
        else:
            setattr(p, k, v)
    return p


@pytest.mark.parametrize("kw", [
    dict(strn=0), dict(strn=65), dict(N=0), dict(ens=3), dict(precision=2), dict(alpha=-0.1),
    dict(m=(11, 8, 8)),                   # mesh size with a prime factor above 7
    dict(m=(8, 8, 0)),
    dict(f=1.5), dict(f=float("nan")),
    dict(fcont=1, f=1.0),                 # junction step past the chain end
    dict(fcont=1, f=0.96),                # homopolymer reaches the junction step
])
def test_create_refuses_bad_problems_before_any_device_call(built_lib, kw):
    """scft_create checks the problem on the host and returns BAD_INPUT
    (never a fallback, never an exit) before it touches a device."""
    h = ctypes.c_void_p()
    rc = S.lib().scft_create(ctypes.byref(_problem(**kw)), ctypes.byref(h))
    assert rc == 3 and not h.value


def test_create_without_a_device_is_unsupported(built_lib):
    """A valid problem with no visible device: SCFT_UNSUPPORTED, no CPU path."""
    code = ("import ctypes, sys; sys.path.insert(0, %r); import scft_string_b200 as S; "
            "from test_abi import _problem; h = ctypes.c_void_p(); "
            "print(S.lib().scft_create(ctypes.byref(_problem()), ctypes.byref(h)))" % os.path.dirname(__file__))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "6"


def test_missing_library_raises(built_lib, monkeypatch, tmp_path):
    monkeypatch.setattr(S, "_lib", None)
    monkeypatch.setattr(S, "LIB_PATH", str(tmp_path / "libscft_b200.so"))
    with pytest.raises(S.ScftError):
        S.lib()
