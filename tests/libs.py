"""Loading the three libraries that speak the LMie C interface, and comparing
their results.

  product()    lmie_b200/liblmie_b200.so   -- the CUDA product
  oracle()     oracle/liblmie_oracle.so    -- CPU restatement (checker)
  reference()  oracle/_ref/liblmie_ref.so  -- the reference itself, compiled
                                              from its sources (None when the
                                              reference tree was not available
                                              at build time)
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Dict, Optional

import numpy as np

from lmie_b200 import abi

ROOT = Path(__file__).resolve().parent.parent
PRODUCT_SO = ROOT / "lmie_b200" / "liblmie_b200.so"
ORACLE_SO = ROOT / "oracle" / "liblmie_oracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "liblmie_ref.so"
GOLDEN = ROOT / "tests" / "golden"

_cache: Dict[str, C.CDLL] = {}


def _load(key, path, binder):
    if key not in _cache:
        lib = C.CDLL(str(path))
        binder(lib)
        _cache[key] = lib
    return _cache[key]


def product() -> C.CDLL:
    if not PRODUCT_SO.exists():
        raise RuntimeError(f"{PRODUCT_SO} is missing: run `python -m lmie_b200.build`")
    return _load("product", PRODUCT_SO, abi.bind_product_like)


def oracle() -> C.CDLL:
    if not ORACLE_SO.exists():
        import subprocess
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True,
                       stdout=subprocess.DEVNULL)
    return _load("oracle", ORACLE_SO, abi.bind_oracle)


def reference() -> Optional[C.CDLL]:
    if not REF_SO.exists():
        return None
    return _load("reference", REF_SO, abi.bind_product_like)


def run_product(case: abi.Case) -> abi.Result:
    return abi.solve(product(), case)


def run_oracle(case: abi.Case) -> abi.Result:
    return abi.solve(oracle(), case, kind="oracle")


def run_reference(case: abi.Case, n_threads: int = 1) -> Optional[abi.Result]:
    lib = reference()
    if lib is None:
        return None
    return abi.solve(lib, case, n_threads=n_threads)


# ---------------------------------------------------------------------------
# comparison (max-norm relative error per output array)
# ---------------------------------------------------------------------------
ARRAYS = ("gc", "lc", "pf", "gc_l", "lc_l", "pf_l", "save1", "save2")


def relmax(a, b) -> float:
    """max|a - b| / max|b| over an array (b is the reference)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return float("inf")
    if b.size == 0:
        return 0.0
    den = float(np.max(np.abs(b)))
    num = float(np.max(np.abs(a - b)))
    if den == 0.0:
        return num
    return num / den


def rel_scalar(a: float, b: float) -> float:
    if a == b:
        return 0.0
    return abs(a - b) / max(abs(b), 1e-300)


def compare(got: abi.Result, want: abi.Result, n_coef_slack: bool = True) -> Dict[str, float]:
    """Per-output errors of `got` against `want`.  GSF/Legendre arrays are
    compared over the shorter n_coef (a coefficient at the truncation
    threshold may flip the count by one)."""
    err: Dict[str, float] = {}
    for k, v in want.scalars.items():
        err[k] = rel_scalar(got.scalars[k], v)
    for k, v in want.scalars_l.items():
        err[k + "_l"] = relmax(got.scalars_l[k], v)
    nc = min(got.n_coef, want.n_coef)
    err["n_coef"] = float(abs(got.n_coef - want.n_coef))
    for name in ARRAYS:
        w = getattr(want, name)
        g = getattr(got, name)
        if w is None:
            continue
        if g is None:
            err[name] = float("inf")
            continue
        if name in ("gc", "lc"):
            g, w = g[:, :nc], w[:, :nc]
        elif name in ("gc_l", "lc_l"):
            g, w = g[:, :, :nc], w[:, :, :nc]
        err[name] = relmax(g, w)
    return err


def result_to_npz(res: abi.Result) -> Dict[str, np.ndarray]:
    d: Dict[str, np.ndarray] = {"n_coef": np.array(res.n_coef)}
    for k, v in res.scalars.items():
        d["s_" + k] = np.array(v)
    for k, v in res.scalars_l.items():
        d["l_" + k] = np.asarray(v)
    for name in ARRAYS + ("theta",):
        v = getattr(res, name)
        if v is not None:
            d[name] = np.asarray(v)
    return d


def npz_to_result(z) -> abi.Result:
    r = abi.Result(rc=0, n_coef=int(z["n_coef"]))
    for k in z.files:
        if k.startswith("s_"):
            r.scalars[k[2:]] = float(z[k])
        elif k.startswith("l_"):
            r.scalars_l[k[2:]] = np.asarray(z[k])
        elif k in ARRAYS or k == "theta":
            setattr(r, k, np.asarray(z[k]))
    return r


def golden(name: str) -> Optional[abi.Result]:
    p = GOLDEN / f"ref_{name}.npz"
    if not p.exists():
        return None
    with np.load(p) as z:
        return npz_to_result(z)
