"""Generates tests/golden/cli/<name>/ from the reference's calllmie.

    make -C oracle ref-cli          # oracle/_ref/calllmie_ref from the reference sources
    python tests/golden/make_cli_golden.py

Each case of tests/cli_cases.py runs in its own output directory; the files
it writes and its standard output (stdout.txt) are the fixture.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))

from cli_cases import CLI_CASES  # noqa: E402

EXE = ROOT / "oracle" / "_ref" / "calllmie_ref"
OUT = ROOT / "tests" / "golden" / "cli"


def main() -> int:
    if not EXE.exists():
        print(f"{EXE} missing: run `make -C oracle ref-cli` first", file=sys.stderr)
        return 1
    for name, args in CLI_CASES.items():
        d = OUT / name
        if d.exists():
            shutil.rmtree(d)
        d.mkdir(parents=True)
        p = subprocess.run([str(EXE)] + args, cwd=d, capture_output=True, text=True)
        if p.returncode != 0:
            print(f"{name}: reference calllmie failed:\n{p.stderr}", file=sys.stderr)
            return 1
        (d / "stdout.txt").write_text(p.stdout)
        print(name, sorted(f.name for f in d.iterdir()))
    return 0


if __name__ == "__main__":
    sys.exit(main())
