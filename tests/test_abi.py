"""The C-ABI library builds for sm_100a, loads, and exports every function
include/scft_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

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
