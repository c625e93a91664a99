"""ctypes mirror of the drop-in C ABI declared in include/lmie_interface.h.

The two structs keep the reference field order byte for byte
(reference src/lmie_interface.h:20-101), so the same ctypes classes drive any
library that exports the LMie interface: liblmie_b200.so (this package), and,
in tests only, the reference library and the CPU oracle.

`Case` is a plain-Python description of one polydisperse problem; `call`
fills an `lmie_in_data`, runs a library's solve entry point and returns every
output as numpy arrays (`Result`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

PD = C.POINTER(C.c_double)
PPD = C.POINTER(PD)
PPPD = C.POINTER(PPD)

# lmieb_reduce_fn (include/lmie_b200.h): int (*)(double *buf, long long count, void *stream, void *ctx)
REDUCE_FN = C.CFUNCTYPE(C.c_int, PD, C.c_longlong, C.c_void_p, C.c_void_p)

# enum size_dist_type (reference misc/rtutil_size_dist.h:22-34); order is ABI.
SIZE_DIST = {
    "none": 0,
    "modified_gamma": 1,
    "log_normal": 2,
    "power_law": 3,
    "gamma": 4,
    "modified_power_law": 5,
    "modified_bimodal_log_normal": 6,
    "exponential": 7,
    "mono": 8,
}

DERIV_INPUTS = ("lambda", "mr", "mi", "a1", "a2", "a3", "a4", "a5", "r1", "r2")


class lmie_in_data(C.Structure):
    _fields_ = [
        ("save_control", C.c_int),
        ("calc_gc", C.c_int),
        ("calc_lc", C.c_int),
        ("calc_pf", C.c_int),
        ("dist_type", C.c_int),
        ("n_int1", C.c_int),
        ("n_int2", C.c_int),
        ("n_quad", C.c_int),
        ("n_angles", C.c_int),
        ("n_derivs", C.c_int),
        ("lambda_", C.c_double),
        ("mr", C.c_double),
        ("mi", C.c_double),
        ("a1", C.c_double),
        ("a2", C.c_double),
        ("a3", C.c_double),
        ("a4", C.c_double),
        ("a5", C.c_double),
        ("r1", C.c_double),
        ("r2", C.c_double),
        ("lambda_l", PD),
        ("mr_l", PD),
        ("mi_l", PD),
        ("a1_l", PD),
        ("a2_l", PD),
        ("a3_l", PD),
        ("a4_l", PD),
        ("a5_l", PD),
        ("r1_l", PD),
        ("r2_l", PD),
        ("accuracy", C.c_double),
    ]


_OUT_SCALARS = ("r1", "r2", "norm", "reff", "veff", "gavg", "vavg", "ravg", "rvw",
                "cext", "csca", "cbak", "g")


class lmie_out_data(C.Structure):
    _fields_ = (
        [("n_coef", C.c_int)]
        + [(n, C.c_double) for n in _OUT_SCALARS]
        + [("gc", PPD), ("lc", PPD), ("theta", PD), ("pf", PPD)]
        + [(n + "_l", PD) for n in _OUT_SCALARS]
        + [("gc_l", PPPD), ("lc_l", PPPD), ("pf_l", PPPD)]
        + [("save1", PPD), ("save2", PPPD)]
    )


@dataclass
class Case:
    """One polydisperse problem, in the units and meaning of lmie_in_data."""

    dist: str = "log_normal"
    lam: float = 0.55
    mr: float = 1.45
    mi: float = 0.001
    a1: float = 0.1
    a2: float = 0.164402
    a3: float = 0.0
    a4: float = 0.0
    a5: float = 0.0
    r1: float = 0.005
    r2: float = 2.0
    n_int1: int = 0
    n_int2: int = 1
    n_quad: int = 200
    n_angles: int = 181
    accuracy: float = 1e-7
    calc_gc: int = 1
    calc_lc: int = 0
    calc_pf: int = 1
    save_control: int = 0
    # derivs[i] maps input name (DERIV_INPUTS) -> d(input)/d(parameter i)
    derivs: List[Dict[str, float]] = field(default_factory=list)

    @property
    def n_derivs(self) -> int:
        return len(self.derivs)


@dataclass
class Result:
    rc: int
    n_coef: int = 0
    scalars: Dict[str, float] = field(default_factory=dict)
    scalars_l: Dict[str, np.ndarray] = field(default_factory=dict)
    gc: Optional[np.ndarray] = None      # [6, n_coef]
    lc: Optional[np.ndarray] = None
    theta: Optional[np.ndarray] = None
    pf: Optional[np.ndarray] = None      # [6, n_angles]
    gc_l: Optional[np.ndarray] = None    # [nd, 6, n_coef]
    lc_l: Optional[np.ndarray] = None
    pf_l: Optional[np.ndarray] = None    # [nd, 6, n_angles]
    save1: Optional[np.ndarray] = None   # [4, n_qsize]
    save2: Optional[np.ndarray] = None   # [4, n_qsize, n_qang]


class InputBlock:
    """Owns an lmie_in_data and the derivative arrays it points at."""

    def __init__(self, case: Case):
        nd = case.n_derivs
        self.arrays = {}
        self.s = lmie_in_data()
        s = self.s
        s.save_control = case.save_control
        s.calc_gc, s.calc_lc, s.calc_pf = case.calc_gc, case.calc_lc, case.calc_pf
        s.dist_type = SIZE_DIST[case.dist] if isinstance(case.dist, str) else int(case.dist)
        s.n_int1, s.n_int2, s.n_quad = case.n_int1, case.n_int2, case.n_quad
        s.n_angles, s.n_derivs = case.n_angles, nd
        s.lambda_, s.mr, s.mi = case.lam, case.mr, case.mi
        s.a1, s.a2, s.a3, s.a4, s.a5 = case.a1, case.a2, case.a3, case.a4, case.a5
        s.r1, s.r2 = case.r1, case.r2
        s.accuracy = case.accuracy
        for name in DERIV_INPUTS:
            arr = np.zeros(max(nd, 1), dtype=np.float64)
            for i, d in enumerate(case.derivs):
                arr[i] = float(d.get(name, 0.0))
            self.arrays[name] = arr
            setattr(s, name + "_l", arr.ctypes.data_as(PD))


def _vec(p, n) -> np.ndarray:
    if not p or n <= 0:
        return np.zeros(0)
    return np.ctypeslib.as_array(p, shape=(n,)).copy()


def _rows2(pp, rows, cols) -> np.ndarray:
    # row pointers over one contiguous block: rows are pp[0] + i*cols
    return np.ctypeslib.as_array(pp[0], shape=(rows, cols)).copy()


def _rows3(ppp, a, b, c) -> np.ndarray:
    return np.ctypeslib.as_array(ppp[0][0], shape=(a, b, c)).copy()


def read_output(case: Case, out: lmie_out_data, max_coef: int, n_qsize: int = 0,
                n_qang: int = 0) -> Result:
    nd = case.n_derivs
    r = Result(rc=0, n_coef=out.n_coef)
    for n in _OUT_SCALARS:
        r.scalars[n] = getattr(out, n)
        if nd > 0:
            r.scalars_l[n] = _vec(getattr(out, n + "_l"), nd)
    nc = max(out.n_coef, 0)
    if case.calc_gc and out.gc:
        r.gc = _rows2(out.gc, 6, max_coef)[:, :nc]
        if nd > 0:
            r.gc_l = _rows3(out.gc_l, nd, 6, max_coef)[:, :, :nc]
    if case.calc_lc and out.lc:
        r.lc = _rows2(out.lc, 6, max_coef)[:, :nc]
        if nd > 0:
            r.lc_l = _rows3(out.lc_l, nd, 6, max_coef)[:, :, :nc]
    if case.calc_pf and out.pf:
        r.theta = _vec(out.theta, case.n_angles)
        r.pf = _rows2(out.pf, 6, case.n_angles)
        if nd > 0:
            r.pf_l = _rows3(out.pf_l, nd, 6, case.n_angles)
    if case.save_control == 1 and out.save1 and n_qsize > 0:
        r.save1 = _rows2(out.save1, 4, n_qsize)
        if n_qang > 0:
            r.save2 = _rows3(out.save2, 4, n_qsize, n_qang)
    return r


def n_qsize(case: Case) -> int:
    """Number of radius nodes (reference misc/rtutil_size_dist.c:20-49)."""
    if case.dist == "mono":
        return 1
    if case.dist == "modified_power_law":
        return case.n_int1 * case.n_quad + case.n_int2 * case.n_quad
    return case.n_int2 * case.n_quad


def solve(lib: C.CDLL, case: Case, n_threads: int = 1, kind: str = "lmie", use_mpi: int = 0) -> Result:
    """Run one case through `lib` and copy every output into numpy arrays.

    kind "lmie": the library exports lmie_solution/lmie_out_free (the product
    and the reference); kind "oracle": oracle_solution/oracle_out_free.
    use_mpi is lmie_solution's last argument (radius sharing with the
    library's registered group).
    """
    blk = InputBlock(case)
    out = lmie_out_data()
    if kind == "oracle":
        max_coef = lib.oracle_calc_max_coef(C.c_double(case.lam), blk.s.dist_type,
                                            C.c_double(case.a1), C.c_double(case.a2),
                                            C.c_double(case.a3), C.c_double(case.r1),
                                            C.c_double(case.r2))
        rc = lib.oracle_solution(C.byref(blk.s), C.byref(out), 1)
    else:
        max_coef = lib.lmie_calc_max_coef(case.lam, blk.s.dist_type, case.a1, case.a2,
                                          case.a3, case.r1, case.r2)
        rc = lib.lmie_solution(C.byref(blk.s), C.byref(out), 1, 0, n_threads, use_mpi)
    if rc != 0:
        return Result(rc=rc)
    nq = n_qsize(case)
    nqang = 0
    if case.save_control == 1:
        nqang = max_coef if (case.calc_gc or case.calc_lc) else 0
    res = read_output(case, out, max_coef, nq, nqang)
    if kind == "oracle":
        if case.save_control == 1:
            lib.oracle_free_save(C.byref(out))
        lib.oracle_out_free(C.byref(out), 1 if case.n_derivs > 0 else 0)
    else:
        lib.lmie_out_free(C.byref(out), 1 if case.n_derivs > 0 else 0)
    return res


def _bind_share(lib: C.CDLL) -> None:
    lib.lmieb_partial_size.restype = C.c_longlong
    lib.lmieb_partial_size.argtypes = [C.POINTER(lmie_in_data)]
    lib.lmieb_solution_partial.restype = C.c_int
    lib.lmieb_solution_partial.argtypes = [C.POINTER(lmie_in_data), C.c_int, C.c_int, PD, C.c_int]
    lib.lmieb_solution_finish.restype = C.c_int
    lib.lmieb_solution_finish.argtypes = [C.POINTER(lmie_in_data), C.POINTER(lmie_out_data), C.c_int, PD,
                                          C.c_int]


def bind_group(lib: C.CDLL) -> None:
    """Declares the radius-sharing entry points of include/lmie_b200.h."""
    _bind_share(lib)
    lib.lmieb_set_radius_group.restype = C.c_int
    lib.lmieb_set_radius_group.argtypes = [C.c_int, C.c_int, REDUCE_FN, C.c_void_p]
    lib.lmieb_nccl_unique_id.restype = C.c_int
    lib.lmieb_nccl_unique_id.argtypes = [C.c_void_p]
    lib.lmieb_set_radius_group_nccl.restype = C.c_int
    lib.lmieb_set_radius_group_nccl.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.lmieb_get_radius_group.restype = C.c_int
    lib.lmieb_get_radius_group.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]


def solve_partial(lib: C.CDLL, case: Case, rank: int, world: int) -> np.ndarray:
    """lmieb_solution_partial(): the integrals of the radii i % world == rank
    of `case` (lmieb_partial_size() doubles, before normalisation)."""
    _bind_share(lib)
    blk = InputBlock(case)
    acc = np.zeros(lib.lmieb_partial_size(C.byref(blk.s)), dtype=np.float64)
    rc = lib.lmieb_solution_partial(C.byref(blk.s), rank, world, acc.ctypes.data_as(PD), 0)
    if rc != 0:
        raise RuntimeError(f"lmieb_solution_partial failed ({rc})")
    return acc


def solve_finish(lib: C.CDLL, case: Case, acc: np.ndarray) -> Result:
    """lmieb_solution_finish(): the solve of `case` from the integrals summed
    over all ranks."""
    _bind_share(lib)
    blk = InputBlock(case)
    acc = np.ascontiguousarray(acc, dtype=np.float64)
    if acc.size != lib.lmieb_partial_size(C.byref(blk.s)):
        raise ValueError("acc has the wrong size for this case")
    out = lmie_out_data()
    max_coef = lib.lmie_calc_max_coef(case.lam, blk.s.dist_type, case.a1, case.a2, case.a3, case.r1, case.r2)
    rc = lib.lmieb_solution_finish(C.byref(blk.s), C.byref(out), 1, acc.ctypes.data_as(PD), 0)
    if rc != 0:
        return Result(rc=rc)
    res = read_output(case, out, max_coef)
    lib.lmie_out_free(C.byref(out), 1 if case.n_derivs > 0 else 0)
    return res


def bind_oracle(lib: C.CDLL) -> None:
    lib.oracle_solution.restype = C.c_int
    lib.oracle_solution.argtypes = [C.POINTER(lmie_in_data), C.POINTER(lmie_out_data), C.c_int]
    lib.oracle_calc_max_coef.restype = C.c_int
    lib.oracle_calc_max_coef.argtypes = [C.c_double, C.c_int] + [C.c_double] * 5
    lib.oracle_out_free.restype = None
    lib.oracle_out_free.argtypes = [C.POINTER(lmie_out_data), C.c_int]
    lib.oracle_free_save.restype = None
    lib.oracle_free_save.argtypes = [C.POINTER(lmie_out_data)]


def bind_product_like(lib: C.CDLL) -> None:
    lib.lmie_solution.restype = C.c_int
    lib.lmie_solution.argtypes = [C.POINTER(lmie_in_data), C.POINTER(lmie_out_data), C.c_int,
                                  C.c_int, C.c_int, C.c_int]
    lib.lmie_out_free.restype = None
    lib.lmie_out_free.argtypes = [C.POINTER(lmie_out_data), C.c_int]
    lib.lmie_calc_max_coef.restype = C.c_int
    lib.lmie_calc_max_coef.argtypes = [C.c_double, C.c_int] + [C.c_double] * 5


def deriv_unit(*names: str) -> List[Dict[str, float]]:
    """One derivative per name, each with unit perturbation of that input."""
    return [{n: 1.0} for n in names]


PRECISION_FP64 = 0      # LMIEB_PRECISION_FP64
PRECISION_TF32X3 = 1    # LMIEB_PRECISION_TF32X3
PRECISION_INT8 = 2      # LMIEB_PRECISION_INT8


def solve_batch(lib: C.CDLL, cases: Sequence[Case], n_threads: int = 8,
                precision: int = PRECISION_FP64) -> List[Result]:
    """Solve many cases with one lmie_solution_batch2() call."""
    n = len(cases)
    blocks = [InputBlock(c) for c in cases]
    ins = (lmie_in_data * n)(*[b.s for b in blocks])
    outs = (lmie_out_data * n)()
    f = lib.lmie_solution_batch2
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.POINTER(lmie_in_data), C.POINTER(lmie_out_data), C.c_int, C.c_int, C.c_int,
                  C.c_int]
    rc = f(n, ins, outs, 1, 0, n_threads, precision)
    if rc != 0:
        return [Result(rc=rc) for _ in cases]
    res = []
    for i, c in enumerate(cases):
        mc = lib.lmie_calc_max_coef(c.lam, ins[i].dist_type, c.a1, c.a2, c.a3, c.r1, c.r2)
        nqang = mc if (c.save_control == 1 and (c.calc_gc or c.calc_lc)) else 0
        res.append(read_output(c, outs[i], mc, n_qsize(c), nqang))
        lib.lmie_out_free(C.byref(outs[i]), 1 if c.n_derivs > 0 else 0)
    return res
