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
        _lib = lib
    return _lib


def solve(case: abi.Case) -> abi.Result:
    """One polydisperse solve through lmie_solution()."""
    return abi.solve(library(), case)


N_STAGES = 9
STAGES = ("upload", "mie_coefficients", "cross_sections", "angular", "normalise",
          "gsf_expansion", "legendre_expansion", "user_angles", "download")
