"""Failure paths, taken without a GPU fault.

- The bounded waits of the tensor-core kernels: the int8 self-test with a
  short wait limit and its first chunk's products withheld, so the wait for
  them runs out (nothing will ever arrive on that barrier): the call returns
  -1, the kernel has released its tensor memory (the next self-tests, which
  allocate all 512 columns, run and pass) and the device keeps working.
- Host-side fault injection (LMIEB_FAULT): the device arena, the pinned
  staging buffer, a sub-batch's input upload and the instantiation of a
  captured kernel sequence fail as their CUDA calls would; the call returns
  -1, nothing leaks (the library's holdings and the device's free memory come
  back to what they were), and the next call gives the same bits as before.
"""
import ctypes as C
import os

import numpy as np
import pytest

import libs
from cases import all_cases
from lmie_b200 import abi, workloads

pytestmark = pytest.mark.gpu


def _lib():
    lib = libs.product()
    lib.lmieb_oz_selftest.restype = C.c_int
    lib.lmieb_oz_selftest.argtypes = [C.c_int, C.POINTER(C.c_double)]
    lib.lmieb_oz_selftest_wait.restype = C.c_int
    lib.lmieb_oz_selftest_wait.argtypes = [C.c_int, C.c_longlong, C.c_int, C.POINTER(C.c_double)]
    lib.lmieb_memory.restype = C.c_int
    lib.lmieb_memory.argtypes = [C.POINTER(C.c_longlong)]
    return lib


def _memory(lib):
    m = (C.c_longlong * 4)()
    assert lib.lmieb_memory(m) == 0
    return {"free": m[0], "total": m[1], "device": m[2], "pinned": m[3]}


class _fault:
    def __init__(self, sites):
        self.sites = sites

    def __enter__(self):
        os.environ["LMIEB_FAULT"] = self.sites

    def __exit__(self, *exc):
        os.environ.pop("LMIEB_FAULT", None)


def _same(a, b):
    for x, y in zip(a, b):
        assert x.rc == 0 and y.rc == 0 and x.n_coef == y.n_coef
        for name in ("gc", "pf", "gc_l", "pf_l"):
            assert np.array_equal(getattr(x, name), getattr(y, name)), name
        assert x.scalars == y.scalars


def test_bounded_wait_runs_out_and_releases_tensor_memory():
    lib = _lib()
    e = C.c_double(-1.)
    for _ in range(2):
        # ~1 ms of waiting for products that are never issued
        assert lib.lmieb_oz_selftest_wait(32, 1 << 21, 1, C.byref(e)) == -1
        assert lib.lmieb_oz_selftest(256, C.byref(e)) == 0 and 0. <= e.value < 1e-11, e.value
    # the same short limit is enough when the products are issued
    assert lib.lmieb_oz_selftest_wait(256, 1 << 21, 0, C.byref(e)) == 0 and e.value < 1e-11
    # and the product path is intact
    case = all_cases()["c2"]
    (ref,) = abi.solve_batch(lib, [case], precision=abi.PRECISION_FP64)
    (got,) = abi.solve_batch(lib, [case], precision=abi.PRECISION_INT8)
    assert got.rc == 0 and got.n_coef == ref.n_coef
    assert libs.compare(got, ref)["pf_l"] < 1e-9


def test_selftest_wait_limit_is_checked():
    lib = _lib()
    e = C.c_double(-1.)
    assert lib.lmieb_oz_selftest_wait(32, 0, 0, C.byref(e)) == -1
    assert lib.lmieb_oz_selftest_wait(32, (1 << 31) + 1, 0, C.byref(e)) == -1


@pytest.mark.parametrize("site", ["alloc", "pinned", "h2d"])
@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_INT8])
def test_injected_failure_propagates_without_leaks(site, precision):
    lib = _lib()
    cases = workloads.batched_uneven(24)
    before = abi.solve_batch(lib, cases, n_threads=4, precision=precision)
    m0 = _memory(lib)
    with _fault(site):
        failed = abi.solve_batch(lib, cases, n_threads=4, precision=precision)
    assert all(r.rc == -1 for r in failed)
    after = abi.solve_batch(lib, cases, n_threads=4, precision=precision)
    _same(after, before)
    m1 = _memory(lib)
    # the failed buffer was rebuilt at this batch's size (no larger than what
    # earlier, larger batches left), and what the library let go of is back
    # on the device: nothing was lost on the way
    released = m0["device"] - m1["device"]
    assert released >= 0 and m1["pinned"] <= m0["pinned"], (m0, m1)
    assert abs((m1["free"] - m0["free"]) - released) <= 4 << 20, (m0, m1)


def test_injected_failure_at_one_of_several_sites():
    """A comma-separated list; names that are not sites change nothing."""
    lib = _lib()
    cases = workloads.batched_uneven(8)
    with _fault("nothing,h2d"):
        assert all(r.rc == -1 for r in abi.solve_batch(lib, cases, n_threads=4))
    with _fault("nothing,graph2"):
        assert all(r.rc == 0 for r in abi.solve_batch(lib, cases, n_threads=4))


def test_injected_graph_failure():
    lib = _lib()
    lib.lmieb_rerun_device.restype = C.c_int
    cases = workloads.batched_uneven(16)
    ms = C.c_double()
    st = (C.c_double * 16)()
    assert lib.lmieb_set_pipeline(1) == 0
    try:
        assert all(r.rc == 0 for r in abi.solve_batch(lib, cases, n_threads=4))
        with _fault("graph"):
            assert lib.lmieb_rerun_device(1, 0, C.byref(ms), st) == -1
        assert lib.lmieb_rerun_device(2, 0, C.byref(ms), st) == 0 and ms.value > 0.
    finally:
        lib.lmieb_set_pipeline(0)
