"""The C host layer's batch flow (lmie_b200/csrc/host_api.c) on the CPU, with
the device layer replaced by a recording stub (tests/host_batch_check.cc):
every case hands the device the same per-radius arrays whether the call is
cut into 1, 3 or 4 parts and when its scratch blocks are reused from the
pool, for every size distribution; the stub's results land in the right
callers' arrays; a single solve prepares what the batch prepares, and so
does the Fortran entry on column-major arrays, whose results land at their
column-major places; save_control 1 returns the kernels and 2 reads them
with its w2 weights; a process
of a radius group gets radii rank, rank + world, ...; a case the host
rejects fails the call and the next call is whole again."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "lmie_b200" / "csrc"


def _build_and_run(tmp_path, flags):
    cc, cxx = shutil.which("gcc"), shutil.which("g++")
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    objs = []
    for src in ("host_api.c", "host_dist.c", "host_fortran.c"):
        obj = tmp_path / (src + ".o")
        subprocess.run([cc, *flags, "-std=gnu99", "-fPIC", *inc, "-c", str(CSRC / src), "-o", str(obj)],
                       check=True)
        objs.append(str(obj))
    exe = tmp_path / "host_batch_check"
    subprocess.run([cxx, *flags, "-std=c++17", "-pthread", *inc, str(ROOT / "tests" / "host_batch_check.cc"),
                    *objs, "-lm", "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr


def test_batch_host_layer_with_a_stubbed_device(tmp_path):
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("no C/C++ compiler")
    _build_and_run(tmp_path, ["-O2"])


def test_batch_host_layer_under_address_sanitizer(tmp_path):
    """The same check with out-of-bounds accesses, use after free and leaks
    of the host layer reported by AddressSanitizer."""
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("no C/C++ compiler")
    probe = subprocess.run(["gcc", "-fsanitize=address", "-x", "c", "-", "-o", str(tmp_path / "probe")],
                           input="int main(void) { return 0; }", capture_output=True, text=True)
    if probe.returncode != 0:
        pytest.skip("no AddressSanitizer")
    _build_and_run(tmp_path, ["-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer"])
