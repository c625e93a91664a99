"""The drop-in boundary, checked without a GPU: the library loads, exports
every function include/*.h declares, keeps the reference's struct layout,
and its host-only helpers behave like the reference's."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

import libs
from conftest import HAS_GPU
from lmie_b200 import abi, build


def _declared():
    return build.exported_symbols()


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(libs.PRODUCT_SO)],
                         stdout=subprocess.PIPE, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in _declared() if s not in exported]
    assert not missing, missing
    lib = libs.product()
    for s in _declared():
        assert hasattr(lib, s), s


def test_reference_symbols_are_all_declared():
    """Every entry point of the reference interface (src/lmie_interface.h,
    interfaces/lmie_int_util.c, the size-distribution name helpers) is here."""
    want = ["lmie_calc_max_coef", "lmie_in_alloc", "lmie_in_free", "lmie_out_alloc",
            "lmie_out_free", "lmie_in_zero_derivs", "lmie_solution", "lmie_solution2",
            "lmie_solution2_l", "lmie_solution_slave", "size_dist_code", "size_dist_name",
            "size_dist_code_", "lmie_calc_max_coef_", "lmie_solution2_", "lmie_solution2_l_"]
    assert set(want) <= set(_declared())


def test_struct_layout_matches_reference():
    # 10 ints, 10 doubles, 10 pointers, 1 double (reference src/lmie_interface.h:20-57)
    assert C.sizeof(abi.lmie_in_data) == 10 * 4 + 10 * 8 + 10 * 8 + 8
    assert abi.lmie_in_data.lambda_.offset == 40
    assert abi.lmie_in_data.accuracy.offset == 200
    # int + pad, 13 doubles, 4 pointers, 13 pointers, 3 pointers, 2 pointers
    assert C.sizeof(abi.lmie_out_data) == 8 + 13 * 8 + 4 * 8 + 13 * 8 + 3 * 8 + 2 * 8
    ref = libs.reference()
    if ref is not None:
        # the same struct drives the reference library (see test_oracle_pins)
        assert ref.lmie_calc_max_coef(0.55, 2, 0.1, 0.16, 0.0, 0.005, 2.0) == 84


def test_calc_max_coef_matches_reference():
    lib = libs.product()
    orc = libs.oracle()
    for lam, r2 in [(0.55, 2.0), (0.865, 60.0), (0.34, 400.0), (2.25, 50.0), (10.0, 0.05)]:
        got = lib.lmie_calc_max_coef(lam, 2, 0.1, 0.16, 0.0, 0.005, r2)
        want = orc.oracle_calc_max_coef(lam, 2, 0.1, 0.16, 0.0, 0.005, r2)
        assert got == want
    # power law: the range comes from the root finder, not from r1/r2
    got = lib.lmie_calc_max_coef(0.6, 3, 0.5, 0.2, 0.0, 0.0, 0.0)
    want = orc.oracle_calc_max_coef(0.6, 3, 0.5, 0.2, 0.0, 0.0, 0.0)
    assert got == want and got > 0


def test_size_dist_names():
    lib = libs.product()
    lib.size_dist_code.restype = C.c_int
    lib.size_dist_code.argtypes = [C.c_char_p]
    lib.size_dist_name.restype = C.c_char_p
    lib.size_dist_name.argtypes = [C.c_int]
    for name, code in abi.SIZE_DIST.items():
        assert lib.size_dist_code(name.encode()) == code
        assert lib.size_dist_name(code).decode() == name
    assert lib.size_dist_code(b"not_a_distribution") == -1
    assert lib.size_dist_name(99) is None
    lib.size_dist_code_.restype = C.c_int
    assert lib.size_dist_code_(C.c_char_p(b"gamma")) == 4


def test_in_alloc_zero_free_and_out_alloc_layout():
    lib = libs.product()
    lib.lmie_in_alloc.argtypes = [C.POINTER(abi.lmie_in_data), C.c_int]
    lib.lmie_in_zero_derivs.argtypes = [C.POINTER(abi.lmie_in_data), C.c_int]
    lib.lmie_in_free.argtypes = [C.POINTER(abi.lmie_in_data), C.c_int]
    lib.lmie_out_alloc.argtypes = [C.POINTER(abi.lmie_in_data), C.POINTER(abi.lmie_out_data), C.c_int]
    s = abi.lmie_in_data()
    assert lib.lmie_in_alloc(C.byref(s), 3) == 0
    for f in abi.DERIV_INPUTS:
        getattr(s, f + "_l")[2] = 7.0
    lib.lmie_in_zero_derivs(C.byref(s), 3)
    for f in abi.DERIV_INPUTS:
        assert [getattr(s, f + "_l")[i] for i in range(3)] == [0.0, 0.0, 0.0]
    s.calc_gc, s.calc_lc, s.calc_pf, s.n_angles, s.n_derivs = 1, 1, 1, 5, 3
    o = abi.lmie_out_data()
    assert lib.lmie_out_alloc(C.byref(s), C.byref(o), 10) == 0
    # row pointers over one contiguous block (reference misc/gutil_alloc.c)
    base = C.cast(o.gc[0], C.c_void_p).value
    for e in range(6):
        assert C.cast(o.gc[e], C.c_void_p).value == base + e * 10 * 8
    base = C.cast(o.pf_l[0][0], C.c_void_p).value
    for d in range(3):
        for e in range(6):
            assert C.cast(o.pf_l[d][e], C.c_void_p).value == base + (d * 6 + e) * 5 * 8
    lib.lmie_out_free(C.byref(o), 1)
    lib.lmie_in_free(C.byref(s), 1)


def test_input_errors_return_minus_one():
    """calc_pf without gc/lc and an unknown distribution are rejected on the
    host, before any device work (reference src/lmie_interface.c:404-408,
    misc/rtutil_size_dist.c:616-619)."""
    lib = libs.product()
    r = abi.solve(lib, abi.Case(calc_gc=0, calc_lc=0, calc_pf=1))
    assert r.rc == -1
    r = abi.solve(lib, abi.Case(dist=99))
    assert r.rc == -1


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    """Without a GPU the solve fails loudly instead of computing on the CPU."""
    r = abi.solve(libs.product(), abi.Case())
    assert r.rc == -1


def test_slave_entry_reports_no_mpi():
    lib = libs.product()
    lib.lmie_solution_slave.restype = C.c_int
    assert lib.lmie_solution_slave() == -1


def test_user_angle_part_argument_checks():
    """Orders per block of the user-angle phase matrix: multiples of 64 from
    64 to 4096 (no GPU needed to set it)."""
    import ctypes as C
    lib = libs.product()
    lib.lmieb_set_user_angle_part.argtypes = [C.c_int]
    keep = lib.lmieb_get_user_angle_part()
    try:
        for bad in (0, 32, 100, 4160, -64):
            assert lib.lmieb_set_user_angle_part(bad) == -1, bad
        assert lib.lmieb_get_user_angle_part() == keep
        assert lib.lmieb_set_user_angle_part(128) == 0 and lib.lmieb_get_user_angle_part() == 128
    finally:
        lib.lmieb_set_user_angle_part(keep)
