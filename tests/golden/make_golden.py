"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run in a tree where the reference sources are available (it reads them, it
never copies them):

    make -C oracle ref              # compiles the reference into oracle/_ref/
    python tests/golden/make_golden.py

Writes
  ref_<case>.npz    every output of the reference's lmie_solution (single
                    thread, full double precision) for each case of
                    tests/cases.py, together with the case definition;
  example_out.npz   the values printed in the reference's golden output
                    examples/example.out (7 significant digits), parsed;
  ref_<case>.npz    likewise for the cases of tests/cases.py large_cases()
                    (size parameters 500 - 5000; about half a minute of
                    reference CPU time in all).
"""
from __future__ import annotations

import dataclasses
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from cases import all_cases, example_case, large_cases  # noqa: E402
import libs  # noqa: E402

REF_TREE = Path(os.environ.get("LMIE_REFERENCE", "/root/reference"))
OUT = ROOT / "tests" / "golden"


def case_json(case) -> str:
    return json.dumps(dataclasses.asdict(case), sort_keys=True)


def parse_example_out(path: Path) -> dict:
    """examples/example.out: 5 blocks (value, d/dmr, d/dmi, d/da1, d/da2), each
    with 10 scalars, n_coef, an n_coef x 6 GSF table and a 181 x 7 phase
    matrix table."""
    text = path.read_text().splitlines()
    blocks = []
    i = 0
    num = r"[-+]?\d\.\d+E[-+]\d+"
    while i < len(text):
        if text[i].startswith("reff"):
            b = {}
            for _ in range(10):
                k, v = text[i].split("=")
                b[k.strip()] = float(v)
                i += 1
            b["n_coef"] = int(text[i].split("=")[1])
            i += 1
            while not text[i].startswith("-----"):
                i += 1
            i += 1
            gc = []
            while i < len(text) and re.match(r"^\s*" + num, text[i]):
                gc.append([float(v) for v in re.findall(num, text[i])])
                i += 1
            while not text[i].startswith("-----"):
                i += 1
            i += 1
            pf = []
            while i < len(text) and re.match(r"^\s*" + num, text[i]):
                pf.append([float(v) for v in re.findall(num, text[i])])
                i += 1
            b["gc"] = np.array(gc).T          # [6, n_coef]
            b["pf"] = np.array(pf).T          # [7, n_angles]: theta then 6 elements
            blocks.append(b)
        else:
            i += 1
    d = {}
    keys = ["reff", "veff", "gavg", "vavg", "ravg", "rvw", "cext", "csca", "cbak", "g"]
    d["scalars"] = np.array([[b[k] for k in keys] for b in blocks])
    d["scalar_names"] = np.array(keys)
    d["n_coef"] = np.array(blocks[0]["n_coef"])
    d["gc"] = np.stack([b["gc"] for b in blocks])            # [5, 6, n_coef]
    d["theta"] = blocks[0]["pf"][0]
    d["pf"] = np.stack([b["pf"][1:] for b in blocks])        # [5, 6, n_angles]
    d["case"] = np.array(case_json(example_case()))
    return d


def main() -> int:
    if not REF_TREE.exists():
        print("reference tree not found; fixtures are generated where it is available")
        return 1
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True,
                   stdout=subprocess.DEVNULL)
    OUT.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(OUT / "example_out.npz",
                        **parse_example_out(REF_TREE / "examples" / "example.out"))
    for name, case in {**all_cases(), **large_cases()}.items():
        res = libs.run_reference(case, n_threads=1)
        assert res is not None and res.rc == 0, name
        d = libs.result_to_npz(res)
        d["case"] = np.array(case_json(case))
        np.savez_compressed(OUT / f"ref_{name}.npz", **d)
        print(f"{name:28s} n_coef={res.n_coef}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
