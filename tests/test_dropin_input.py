"""Input handling of the drop-in program `scft_b200`, checked without a GPU:
with SCFT_DRY_RUN=1 it reads input.dat and the win files, prints the resolved
problem and the start fields, and exits before any device call.  Expected
values restate the reference: readParameters / setParameters
(scft.cu:80-114, 120-251: '#' comments, whitespace-free keys, the first value
of each key, partial m/D/fix lists keep the remaining defaults, unknown keys
ignored), the defaults of main (scft.cu:37-38, 914-916), the win-file
fallback (scft.cu:1057-1078: a file without exactly M lines copies the
previous replica and adds a spring step; a bad win0 is copied from win1) and
the readwin = 0 start (scft.cu:1079-1098)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "scft_string_b200", "scft_b200")


def dry_run(cwd, args=()):
    env = dict(os.environ, SCFT_DRY_RUN="1")
    out = subprocess.run([EXE, *args], cwd=cwd, env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    problem, run, fields = {}, {}, []
    for line in out.stdout.splitlines():
        t = line.split()
        if line.startswith("dryrun problem") or line.startswith("dryrun run"):
            d = problem if t[1] == "problem" else run
            key = None
            for tok in t[2:]:
                if "=" in tok:
                    key, v = tok.split("=")
                    d[key] = [float(v)]
                else:
                    d[key].append(float(tok))
        elif line.startswith("dryrun field"):
            fields.append([float(x) for x in t[3:]])
    return problem, run, np.array(fields), out.stdout


@pytest.fixture
def exe():
    if not os.path.exists(EXE):
        pytest.skip("scft_b200 is not built")
    return EXE


def write_win(path, wm, wp):
    with open(path, "w") as f:
        for a, b in zip(wm, wp):
            f.write(f"{a:.6f} {b:.6f}\n")


def test_defaults_without_input_file(exe, tmp_path):
    p, run, fl, out = dry_run(tmp_path, ["missing.dat"])
    assert "missing.dat not found" in out
    assert p["m"] == [50, 50, 50] and p["D"] == [4, 4, 4] and p["fix"] == [0, 0]
    assert p["N"] == [60] and p["chi"] == [30] and p["f"] == [0.8] and p["alpha"] == [0.1]
    assert p["ens"] == [2] and p["phidb"] == [0] and p["strn"] == [48] and p["dostring"] == [1]
    assert run["readwin"] == [1] and run["justFE"] == [0] and run["nsterp"] == [4000]
    assert run["handover"] == [0] and run["errtol"] == [0]
    assert p["springsteps"] == [48] and len(fl) == 48 and not fl.any()


def test_handover_and_errtol_keys(exe, tmp_path):
    (tmp_path / "input.dat").write_text("precision = 32\nerrtol = 1e-6\nhandover = 2.5e-4\nstrn = 1\n"
                                        "m = 8 8 8\nreadwin = 0\n")
    p, run, fl, out = dry_run(tmp_path)
    assert p["precision"] == [32]
    assert run["errtol"] == [1e-6] and run["handover"] == [2.5e-4]


def test_keys_comments_partial_lists(exe, tmp_path):
    (tmp_path / "input.dat").write_text(
        "# a comment line\n"
        "chi = 15   # trailing comment\n"
        "  f=0.45\n"
        "N = 20.9\n"              # truncated to int as static_cast<int>
        "m = 4 6\n"               # m[2] keeps its default
        "D = 2.5\n"
        "fix = 1\n"
        "unknown key = 3 4\n"     # key 'unknownkey': ignored
        "strn = 2\n"
        "ens=1\n"
        "phi db = 0.8\n"          # whitespace inside a key is removed
        "alpha = 0.2 0.3\n"       # the first value counts
        "\n")
    p, run, fl, _ = dry_run(tmp_path)
    assert p["chi"] == [15] and p["f"] == [0.45] and p["N"] == [20] and p["alpha"] == [0.2]
    assert p["m"] == [4, 6, 50] and p["D"] == [2.5, 4, 4] and p["fix"] == [1, 0]
    assert p["strn"] == [2] and p["ens"] == [1] and p["phidb"] == [0.8]


def test_win_files_and_fallback(exe, tmp_path):
    m = (2, 3, 4)
    M = int(np.prod(m))
    (tmp_path / "input.dat").write_text(f"m = {m[0]} {m[1]} {m[2]}\nstrn = 4\n")
    rng = np.random.default_rng(0)
    w = [(rng.normal(size=M), rng.normal(size=M)) for _ in range(4)]
    write_win(tmp_path / "win0", *w[0])
    write_win(tmp_path / "win1", w[1][0][:-1], w[1][1][:-1])     # one line short: copy of replica 0
    write_win(tmp_path / "win3", *w[3])                           # win2 missing: copy of replica 1
    p, _, fl, out = dry_run(tmp_path)
    assert "win1 is too small: %d." % (M - 1) in out
    assert p["springsteps"] == [2]
    r0 = np.round(w[0][0], 6), np.round(w[0][1], 6)
    r3 = np.round(w[3][0], 6), np.round(w[3][1], 6)
    for ii, (a, b) in enumerate([r0, r0, r0, r3]):
        np.testing.assert_allclose(fl[ii], [a[0], b[0], a.sum(), b.sum()], rtol=1e-12, atol=1e-12)


def test_bad_win0_is_copied_from_win1(exe, tmp_path):
    m = (2, 2, 2)
    (tmp_path / "input.dat").write_text("m = 2 2 2\nstrn = 2\n")
    wm, wp = np.arange(8) * 0.5, -np.arange(8) * 0.25
    write_win(tmp_path / "win1", wm, wp)
    p, _, fl, _ = dry_run(tmp_path)
    assert p["springsteps"] == [1]
    np.testing.assert_allclose(fl[0], fl[1])
    np.testing.assert_allclose(fl[1], [wm[0], wp[0], wm.sum(), wp.sum()])


def test_readwin_zero_start(exe, tmp_path):
    m, chi = (3, 8, 10), 20.0
    (tmp_path / "input.dat").write_text(f"m = {m[0]} {m[1]} {m[2]}\nreadwin = 0\nchi = {chi}\nstrn = 2\n")
    p, _, fl, _ = dry_run(tmp_path)
    assert p["springsteps"] == [0]
    _, Y, Z = np.meshgrid(*[np.arange(k) for k in m], indexing="ij")
    rr = np.sqrt((Z - m[2] / 2.0) ** 2 + (Y - m[1] / 2.0) ** 2)
    w0 = -0.5 * chi * np.exp(-((rr - m[1] / 4.0) / 8.0) ** 2) - 0.5 * chi * np.exp(-((rr - m[1] / 8.0) / 8.0) ** 2)
    np.testing.assert_allclose(fl[0], [w0.ravel()[0], 0.0, w0.sum(), 0.0], rtol=1e-12, atol=1e-12)
    assert not fl[1].any()
