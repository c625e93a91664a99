"""calllmie on liblmie_b200 against the reference's calllmie.

The fixtures under tests/golden/cli/ are the files the reference tool wrote
for the command lines of tests/cli_cases.py (tests/golden/make_cli_golden.py).
The GPU tests run lmie_b200/calllmie with the same command lines and compare
every file: header names and integers exactly, numbers to the 7 significant
digits the format prints (values within 1e-10 of each other may still round
differently in the last digit).  The CPU tests cover the command-line errors,
which exit before any solve.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from cli_cases import CLI_CASES

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "lmie_b200" / "calllmie"
GOLD = ROOT / "tests" / "golden" / "cli"

# printed with %e: 7 significant digits, so neighbours differ by up to 1e-6 relative
RTOL = 1.5e-6
ATOL_REL = 1e-9       # of the largest magnitude in the same column


def run(args, cwd):
    if not EXE.exists():
        pytest.fail(f"{EXE} is not built (python -m lmie_b200.build)")
    return subprocess.run([str(EXE)] + list(args), cwd=cwd, capture_output=True, text=True, timeout=600)


def parse(text: str):
    """(header {name: value string}, table rows) of a scattering text file;
    a bare integer line (row count) goes in the header as 'count'."""
    head, rows = {}, []
    for line in text.splitlines():
        line = line.strip()
        if not line:
            continue
        if "=" in line:
            k, v = line.split("=", 1)
            head[k.strip()] = v.strip()
        elif len(line.split()) == 1 and not rows and "count" not in head:
            head["count"] = line
        else:
            rows.append([float(t) for t in line.split()])
    return head, np.array(rows, dtype=float)


def assert_same_file(got: str, want: str, what: str):
    hg, tg = parse(got)
    hw, tw = parse(want)
    assert list(hg) == list(hw), f"{what}: header fields differ"
    for k in hw:
        a, b = hg[k], hw[k]
        try:
            fa, fb = float(a), float(b)
        except ValueError:
            assert a == b, f"{what}: {k} = {a!r}, reference {b!r}"
            continue
        if k in ("n_int1", "n_int2", "n_quad", "count"):
            assert a == b, f"{what}: {k} = {a}, reference {b}"
        else:
            assert abs(fa - fb) <= RTOL * abs(fb) + 1e-300, f"{what}: {k} = {a}, reference {b}"
    assert tg.shape == tw.shape, f"{what}: table {tg.shape}, reference {tw.shape}"
    if tw.size:
        scale = np.max(np.abs(tw), axis=0, keepdims=True)
        bad = np.abs(tg - tw) > RTOL * np.abs(tw) + ATOL_REL * scale
        assert not bad.any(), f"{what}: {int(bad.sum())} table entries differ, first at {np.argwhere(bad)[0]}"


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CLI_CASES))
def test_cli_matches_reference_tool(name, tmp_path):
    p = run(CLI_CASES[name], tmp_path)
    assert p.returncode == 0, p.stderr
    gold = GOLD / name
    want_files = sorted(f.name for f in gold.iterdir() if f.name != "stdout.txt")
    got_files = sorted(f.name for f in tmp_path.iterdir())
    assert got_files == want_files
    for f in want_files:
        assert_same_file((tmp_path / f).read_text(), (gold / f).read_text(), f"{name}/{f}")
    assert_same_file(p.stdout, (gold / "stdout.txt").read_text(), f"{name}/stdout")


@pytest.mark.gpu
def test_cli_timing_prints_seconds(tmp_path):
    p = run(CLI_CASES["mono_save"][:-2] + ["-timing", "2"], tmp_path)
    assert p.returncode == 0, p.stderr
    assert float(p.stdout.strip().splitlines()[-1]) >= 0.0


def test_cli_help_and_version(tmp_path):
    p = run(["-help"], tmp_path)
    assert p.returncode == 0 and "calllmie" in p.stdout
    p = run(["-version"], tmp_path)
    assert p.returncode == 0 and p.stdout.startswith("calllmie version")


@pytest.mark.parametrize("args, message", [
    ([], "must specify a size distribution with -dist"),
    (["-dist", "gamma", "2", "0.1", "0.01", "6"], "must specify the wavelength with -lambda"),
    (["-dist", "gamma", "2", "0.1", "0.01", "6", "-lambda", "0.5"], "must specify the index of refraction"),
    (["-dist", "gamma", "2", "0.1", "0.01", "6", "-lambda", "0.5", "-m", "1.3", "0"], "-n_int2"),
    (["-dist", "gamma", "2", "0.1", "0.01", "6", "-lambda", "0.5", "-m", "1.3", "0", "-n_int2", "1"], "-n_quad"),
    (["-dist", "mono", "1", "-lambda", "0.5", "-m", "1.3", "0", "-n_int2", "1", "-n_quad", "1",
      "-check_cbak", "1e-5"], "must use -pf when using -check_cbak"),
    (["-dist", "mono", "1", "-lambda", "0.5", "-m", "1.3", "0", "-n_int2", "1", "-n_quad", "1",
      "-check_g", "1e-5"], "must use -pf when using -check_g"),
    (["-dist", "modified_power_law", "-3", "0.1", "2", "-lambda", "0.5", "-m", "1.3", "0"], "-n_int1"),
    (["-dist", "nosuch"], "invalid distribution name"),
    (["-dist_l", "0"], "must specify -dist before -dist_l"),
    (["-m_l", "1", "0"], "Must specifiy -derivs"),
    (["-derivs", "2", "-m_l", "1,0,0", "0,1"], "not consistent with the specified number of derivs: 2"),
    (["-lambda", "x"], "invalid value for -lambda: x"),
    (["-lambda"], "not enough arguments for -lambda"),
])
def test_cli_argument_errors(args, message, tmp_path):
    p = run(args, tmp_path)
    assert p.returncode == 1
    assert message in p.stderr
    assert p.stderr.startswith("ERROR: ")


def test_cli_rejects_unknown_option_and_extra_arguments(tmp_path):
    p = run(["-nosuch"], tmp_path)
    assert p.returncode == 1 and "Invalid option: -nosuch" in p.stdout
    p = run(["extra"], tmp_path)
    assert p.returncode == 1 and "Too many arguments" in p.stdout
