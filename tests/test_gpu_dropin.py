"""The drop-in program `scft_b200` run on the golden cases: every file the
reference program wrote (win<ii>, rhoA_<ii>.vtk, rhocB_<ii>.vtk, FEs, check)
is written by scft_b200 with the same name and layout, and the same numbers
to the printed precision."""
import os
import subprocess

import numpy as np
import pytest

from cases import CASES
from replay import load_fixture
from scft_string_b200.configs import fields, input_dat, win_text

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "scft_string_b200", "scft_b200")


def numbers(txt):
    out = []
    for tok in txt.split():
        try:
            out.append(float(tok))
        except ValueError:
            pass
    return np.array(out)


def _isnum(tok):
    try:
        float(tok)
        return True
    except ValueError:
        return False


def words(txt):
    return [t for t in txt.split() if not _isnum(t)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_files_match_reference(built_lib, tmp_path, name):
    fx = load_fixture(name)
    c = fx["params"]
    wm, wp = fields(c)
    (tmp_path / "input.dat").write_text(input_dat(c) + f"strn = {c['strn']}\nnsterp = {c['nsterp']}\n")
    for ii in range(c["strn"]):
        if ii in c.get("missing", ()):
            continue
        (tmp_path / f"win{ii}").write_text(win_text(wm[ii], wp[ii]))
    p = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    ref_files = fx["files"]
    for fn, ref_txt in ref_files.items():
        path = tmp_path / fn
        assert path.exists(), fn
        got_txt = path.read_text()
        if fn == "check":
            # line 1 holds err3 and FE, uninitialised in the reference at k=0 (scft.cu:772)
            r = numbers(ref_txt)
            g = numbers(got_txt)
            assert r.size == g.size
            assert r[0] == g[0] and abs(r[2] - g[2]) < 1e-9
            assert np.allclose(g[4:], r[4:], rtol=1e-9, atol=1e-11)
            continue
        assert words(got_txt) == words(ref_txt), fn
        r, g = numbers(ref_txt), numbers(got_txt)
        assert r.size == g.size, fn
        if fn.startswith("win"):
            tol = 1.01e-6
        elif fn.endswith(".vtk"):
            tol = 1.01e-4
        else:  # FEs: %lf, %.10lf, %.10lf
            tol = 1.01e-6
        assert np.array_equal(np.isnan(r), np.isnan(g)), fn
        ok = ~np.isnan(r)
        assert np.abs(r[ok] - g[ok]).max() <= tol, (fn, np.abs(r[ok] - g[ok]).max())


def test_dropin_checkpoint_restart(built_lib, tmp_path):
    """`checkpoint = 1` writes fields.ckpt beside the win files; a second run
    with `restart = 1` and no win files starts from it (box and fields) and,
    with justFE = 1 (no string iterations), writes back the same W- fields."""
    name = sorted(CASES)[0]
    c = dict(load_fixture(name)["params"])
    wm, wp = fields(c)
    base = input_dat(c) + f"strn = {c['strn']}\nnsterp = {c['nsterp']}\n"
    a = tmp_path / "a"
    a.mkdir()
    (a / "input.dat").write_text(base + "checkpoint = 1\n")
    for ii in range(c["strn"]):
        (a / f"win{ii}").write_text(win_text(wm[ii], wp[ii]))
    p = subprocess.run([EXE], cwd=a, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert (a / "fields.ckpt").exists()
    b = tmp_path / "b"
    b.mkdir()
    (b / "input.dat").write_text(input_dat(c) + f"strn = {c['strn']}\njustFE = 1\nrestart = 1\n")
    (b / "fields.ckpt").write_bytes((a / "fields.ckpt").read_bytes())
    p = subprocess.run([EXE], cwd=b, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert "fields.ckpt read." in p.stdout
    # the W+ prelude of the second run starts from the restored fields; their
    # W- parts are untouched by it, so W- of every propagated replica matches
    for ii in range(c["strn"]):
        wa, wb = numbers((a / f"win{ii}").read_text()), numbers((b / f"win{ii}").read_text())
        assert wa.size == wb.size
        assert np.abs(wa[0::2] - wb[0::2]).max() <= 1.01e-6, ii


def test_dropin_fp32_handover_reaches_the_fp64_answer(built_lib, tmp_path):
    """`precision = 32` with `handover`: the program iterates in FP32, moves
    the fields to FP64 when errtot falls below the hand-over value (or stops
    improving), continues the same run and stops at `errtol`.  Its final free
    energy equals that of the FP64 run to the same tolerance within 1e-6 kT
    per chain, the FP32 path's accuracy target."""
    name = "plain_c"
    c = dict(load_fixture(name)["params"])
    wm, wp = fields(c)
    fes = {}
    for tag, extra in (("fp64", "precision = 64\n"), ("mixed", "precision = 32\nhandover = 1e-4\n")):
        d = tmp_path / tag
        d.mkdir()
        (d / "input.dat").write_text(input_dat(c) + f"strn = {c['strn']}\nnsterp = 40000\nerrtol = 1e-6\n" + extra)
        for ii in range(c["strn"]):
            (d / f"win{ii}").write_text(win_text(wm[ii], wp[ii]))
        p = subprocess.run([EXE], cwd=d, capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        last = [ln for ln in p.stdout.splitlines() if ln.startswith("error ")][-1]
        errtot = float(last.split()[2].split("/")[0])
        assert errtot <= 1e-6, last
        if tag == "mixed":
            assert "handover to FP64" in p.stdout
        fes[tag] = numbers((d / "FEs").read_text())
        print(tag, last)
    F64, Fmix = fes["fp64"][1::3], fes["mixed"][1::3]
    assert np.abs(F64 - Fmix).max() <= 1e-6
