"""Builds lmie_b200/liblmie_b200.so in-tree.

The host layer (csrc/host_*.c) is compiled as C with gcc, the device code
(csrc/*.cu) with nvcc for sm_100a only, and everything is linked into one
shared library with the CUDA runtime linked statically, so the .so travels
with the source tree and needs only the NVIDIA driver at run time.

    python -m lmie_b200.build          # incremental
    python -m lmie_b200.build --force
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OBJ = HERE / "_build"
LIB = HERE / "liblmie_b200.so"
CLI_SRC = HERE / "cli" / "calllmie.c"
CLI = HERE / "calllmie"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-diag-suppress", "177"]
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu99", "-Wall", "-Wno-unused-function"]


def exported_symbols():
    """Function names declared in include/*.h: exactly the library's exports."""
    import re
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", " ", h.read_text(), flags=re.S)
        # (typedefs of function pointers declare no function)
        for m in re.finditer(r"^(?!typedef\b)[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof") and name not in names:
                names.append(name)
    return names


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblmie_b200")


def _sources():
    c_src = sorted(CSRC.glob("*.c"))
    cu_src = sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return c_src, cu_src, headers


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + proc.stdout)
    return proc.stdout


def build(force: bool = False, verbose: bool = False) -> Path:
    c_src, cu_src, headers = _sources()
    OBJ.mkdir(exist_ok=True)
    nvcc = _nvcc()
    jobs = []
    objs = []
    for src in c_src + cu_src:
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            if src.suffix == ".c":
                cmd = ["gcc"] + CC_FLAGS + ["-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            else:
                cmd = [nvcc] + NVCC_FLAGS + ["-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for out in ex.map(_run, jobs):
                if verbose and out.strip():
                    print(out)
    if force or jobs or _stale(LIB, objs):
        vs = OBJ / "exports.map"
        vs.write_text("{\n  global:\n" + "".join(f"    {n};\n" for n in exported_symbols()) +
                      "  local: *;\n};\n")
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] +
             ["-cudart", "static", "-lm", "-lpthread", "-ldl", "-lrt",
              "-Xlinker", f"--version-script={vs}"])
        os.replace(tmp, LIB)
    # the command-line driver, linked against the library next to it
    if force or _stale(CLI, [CLI_SRC, LIB] + sorted(INCLUDE.glob("*.h"))):
        tmp = CLI.with_suffix(".tmp")
        _run(["gcc"] + CC_FLAGS + ["-I", str(INCLUDE), str(CLI_SRC), "-o", str(tmp), "-L", str(HERE),
                                   "-llmie_b200", "-Wl,-rpath,$ORIGIN", "-lm"])
        os.replace(tmp, CLI)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
