"""B200-native polydisperse Lorenz-Mie solver with LMie's C interface.

The product is the shared library lmie_b200/liblmie_b200.so (C host layer +
sm_100a CUDA kernels); this package locates it, declares its entry points for
ctypes callers (see `abi` for the struct mirror) and builds it (`build`).
There is no CPU fallback: loading fails loudly when the library is missing,
and every solve returns -1 when no sm_100 GPU is usable.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "liblmie_b200.so"
_lib = None


def library() -> C.CDLL:
    """The loaded liblmie_b200.so with argtypes declared."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} not built: run `python -m lmie_b200.build`")
        lib = C.CDLL(str(LIB_PATH))
        abi.bind_product_like(lib)
        lib.lmieb_set_device.argtypes = [C.c_int]
        lib.lmieb_set_timing.argtypes = [C.c_int]
        lib.lmieb_last_timing.argtypes = [C.POINTER(C.c_double), C.c_int]
        lib.lmieb_rerun_device.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]
        lib.lmieb_last_work.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                        C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        lib.lmieb_fp64_peak.argtypes = [C.POINTER(C.c_double)]
        lib.lmieb_device_info.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.lmieb_tc_selftest.argtypes = [C.c_int, C.POINTER(C.c_double)]
        lib.lmieb_oz_selftest.argtypes = [C.c_int, C.POINTER(C.c_double)]
        lib.lmieb_last_host_timing.argtypes = [C.POINTER(C.c_double), C.c_int]
        lib.lmieb_set_pipeline.argtypes = [C.c_int]
        lib.lmieb_set_work_granularity.argtypes = [C.c_int, C.c_double]
        lib.lmieb_get_work_granularity.argtypes = [C.c_int]
        lib.lmieb_get_work_granularity.restype = C.c_double
        lib.lmieb_set_split_segment.argtypes = [C.c_int]
        lib.lmieb_save_cache_stats.argtypes = [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        lib.lmieb_get_split_segment.argtypes = []
        lib.lmieb_set_user_angle_part.argtypes = [C.c_int]
        lib.lmieb_get_user_angle_part.argtypes = []
        abi.bind_group(lib)
        _lib = lib
    return _lib


def solve(case: abi.Case) -> abi.Result:
    """One polydisperse solve through lmie_solution()."""
    return abi.solve(library(), case)


N_STAGES = 9
STAGES = ("upload", "mie_coefficients", "cross_sections", "angular", "normalise",
          "gsf_expansion", "legendre_expansion", "user_angles", "download")


class lmie_bins(C.Structure):
    _fields_ = [("n_bins", C.c_int), ("n_quad", C.c_int),
                ("edges", C.POINTER(C.c_double)), ("weight", C.POINTER(C.c_double))]


class lmie_loss_weights(C.Structure):
    _fields_ = [("c_cext", C.c_double), ("c_csca", C.c_double), ("c_g", C.c_double),
                ("d_p11", C.POINTER(C.c_double)), ("d_p12", C.POINTER(C.c_double))]


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def adjoint(p) -> dict:
    """lmie_solution_adjoint() on a workloads.AdjointProblem: the loss, its
    gradient w.r.t. mr, mi (per wavelength) and the bin weights, and the
    per-wavelength outputs [Cext, Csca, g, P11(theta), P12(theta)]."""
    import numpy as np
    lib = library()
    f = lib.lmie_solution_adjoint
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                  C.POINTER(lmie_bins), C.c_int, C.POINTER(lmie_loss_weights), C.POINTER(C.c_double),
                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L, na = p.n_lambda, p.n_angles
    bins = lmie_bins(p.n_bins, p.n_quad, _dptr(p.edges), _dptr(p.weight))
    w = (lmie_loss_weights * L)()
    for k in range(L):
        w[k] = lmie_loss_weights(p.c[k, 0], p.c[k, 1], p.c[k, 2], _dptr(p.d11[k]), _dptr(p.d12[k]))
    loss = C.c_double()
    gmr, gmi = np.zeros(L), np.zeros(L)
    gw = np.zeros(p.n_bins)
    vals = np.zeros((L, 3 + 2 * na))
    rc = f(L, _dptr(p.lam), _dptr(p.mr), _dptr(p.mi), C.byref(bins), na, w, C.byref(loss),
           _dptr(gmr), _dptr(gmi), _dptr(gw), _dptr(vals))
    if rc != 0:
        raise RuntimeError("lmie_solution_adjoint failed")
    return {"loss": loss.value, "grad_mr": gmr, "grad_mi": gmi, "grad_weight": gw,
            "cext": vals[:, 0], "csca": vals[:, 1], "g": vals[:, 2],
            "p11": vals[:, 3:3 + na], "p12": vals[:, 3 + na:]}
