"""The library's host worker pool (lmie_b200/csrc/host_pool.h) under stress,
on the CPU: a workers' start-up race once left a call waiting for a worker
that had already skipped its job, so the check runs with a time limit."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_host_pool_covers_every_index_and_returns(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "host_pool_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-I", str(ROOT / "lmie_b200" / "csrc"),
                    str(ROOT / "tests" / "host_pool_check.cc"), "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr
