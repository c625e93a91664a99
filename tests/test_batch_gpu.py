"""lmie_solution_batch: many independent cases in batched device launches.

Every case of a batch must give what lmie_solution gives for it alone, and
what the reference gives: the batch changes only how work is grouped on the
device (radius groups, summation order), so results agree to the parity
tolerance."""
import dataclasses
import math

import numpy as np
import pytest

import libs
from cases import all_cases, small_cases
from lmie_b200 import abi, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _assert_close(got, want, tol, label):
    assert got.rc == 0, label
    err = libs.compare(got, want)
    assert err["n_coef"] <= 1, (label, got.n_coef, want.n_coef)
    bad = {k: v for k, v in err.items() if k != "n_coef" and v > tol}
    assert not bad, (label, bad)


def test_batch_of_mixed_cases_matches_reference():
    """Cases with different distributions, derivative layouts and output
    flags in one call: grouped into compatible device batches."""
    names = [n for n in small_cases() if n != "save1"] + ["example", "x1000_few_radii"]
    cases = [all_cases()[n] for n in names]
    got = abi.solve_batch(libs.product(), cases, n_threads=8)
    for n, g in zip(names, got):
        _assert_close(g, libs.golden(n), TOL, n)


def test_uneven_batch_matches_single_solves():
    """A slice of the seeded uneven workload (size parameters 0.2..1000)."""
    cases = workloads.batched_uneven(96)
    got = abi.solve_batch(libs.product(), cases, n_threads=8)
    for i, (c, g) in enumerate(zip(cases, got)):
        _assert_close(g, libs.run_product(c), 1e-12, f"case {i}")


def test_uneven_batch_matches_oracle():
    cases = [c for c in workloads.batched_uneven(64) if 2 * np.pi * c.r2 / c.lam < 60][:12]
    assert len(cases) >= 6
    got = abi.solve_batch(libs.product(), cases, n_threads=4)
    for i, (c, g) in enumerate(zip(cases, got)):
        _assert_close(g, libs.run_oracle(c), TOL, f"case {i}")


def test_batch_with_save_control_case():
    """A save_control case inside a batch is solved on its own."""
    cases = [all_cases()["gamma"], all_cases()["save1"], all_cases()["c1"]]
    got = abi.solve_batch(libs.product(), cases, n_threads=2)
    for n, g in zip(["gamma", "save1", "c1"], got):
        _assert_close(g, libs.golden(n), TOL, n)


def test_batch_reports_bad_case():
    cases = [all_cases()["c1"], dataclasses.replace(all_cases()["c1"], calc_gc=0, calc_lc=0)]
    cases[1] = dataclasses.replace(cases[1], calc_pf=1)
    got = abi.solve_batch(libs.product(), cases, n_threads=2)
    assert got[0].rc == -1


def test_rerun_replays_resident_batch_and_refuses_split_calls():
    """lmieb_rerun_device replays the resident batch as a captured CUDA graph
    only when the last call ran as one part."""
    import ctypes as C
    import lmie_b200
    lib = lmie_b200.library()
    cases = workloads.batched_uneven(64)
    tot = C.c_double()
    st = (C.c_double * lmie_b200.N_STAGES)()
    try:
        lib.lmieb_set_pipeline(1)
        assert all(r.rc == 0 for r in abi.solve_batch(lib, cases, n_threads=4))
        assert lib.lmieb_rerun_device(2, 0, C.byref(tot), st) == 0
        assert tot.value > 0 and st[3] > 0
        lib.lmieb_set_pipeline(4)
        assert all(r.rc == 0 for r in abi.solve_batch(lib, cases, n_threads=4))
        assert lib.lmieb_rerun_device(1, 0, C.byref(tot), st) == -1
    finally:
        lib.lmieb_set_pipeline(0)


def test_pipelined_batch_matches_one_part():
    """Cutting a batch into parts changes only how the work is scheduled: the
    radius groups of the angular stage are planned per part, so the order of
    the partial sums (not the arithmetic) can differ, at round-off level."""
    import lmie_b200
    lib = lmie_b200.library()
    cases = workloads.batched_uneven(96)
    try:
        lib.lmieb_set_pipeline(1)
        one = abi.solve_batch(lib, cases, n_threads=4)
        lib.lmieb_set_pipeline(5)
        many = abi.solve_batch(lib, cases, n_threads=4)
    finally:
        lib.lmieb_set_pipeline(0)
    for i, (a, b) in enumerate(zip(one, many)):
        assert a.rc == 0 and b.rc == 0 and a.n_coef == b.n_coef
        err = libs.compare(b, a)
        bad = {k: v for k, v in err.items() if v > 1e-13}
        assert not bad, (i, bad)


def test_results_in_pieces_match_single_solves():
    """A one-part batch whose results (about 40 MB) come back in several
    pieces of cases, each unpacked while the next is copied: every case as
    when solved alone."""
    import lmie_b200
    lib = lmie_b200.library()
    cases = workloads.batched_uneven(512)
    try:
        lib.lmieb_set_pipeline(1)
        got = abi.solve_batch(lib, cases, n_threads=8)
    finally:
        lib.lmieb_set_pipeline(0)
    for i in range(0, len(cases), 7):
        _assert_close(got[i], libs.run_product(cases[i]), 1e-12, f"case {i}")
    for i, g in enumerate(got):
        assert g.rc == 0 and np.isfinite(g.gc).all() and np.isfinite(g.pf).all(), i


def test_autotune_picks_a_candidate_and_keeps_results():
    import ctypes as C
    import bench
    import lmie_b200
    lib = lmie_b200.library()
    cases = workloads.batched_uneven(64)
    ref = abi.solve_batch(lib, cases, n_threads=4)
    b = bench.CBatch(lib, cases)
    keep = lib.lmieb_get_work_granularity(abi.PRECISION_FP64)
    try:
        got = b.autotune(4, abi.PRECISION_FP64)
        assert got["pipeline_parts"] in (1, 2, 3, 4, 6)
        assert got["angular_items_per_sm"] in (32.0, 64.0, 128.0, 256.0)
        assert got["ms_per_call"] > 0
        assert lib.lmieb_get_user_angle_part() in (128, 256, 512)
        after = abi.solve_batch(lib, cases, n_threads=4)
        for i, (a, r) in enumerate(zip(after, ref)):
            err = libs.compare(a, r)
            assert not {k: v for k, v in err.items() if v > 1e-13}, i
    finally:
        lib.lmieb_set_pipeline(0)
        lib.lmieb_set_work_granularity(abi.PRECISION_FP64, keep)
        lib.lmieb_set_work_granularity(0, C.c_double(4.0))
        lib.lmieb_set_user_angle_part(256)


def test_user_angle_parts_only_reorder_sums():
    """The phase matrix at the user angles with 64 orders per block (large
    cases spread over many blocks whose sums are added in order) and with
    4096 (every case in one block): the same values to round-off."""
    import ctypes as C
    lib = libs.product()
    lib.lmieb_set_user_angle_part.argtypes = [C.c_int]
    cases = [c for c in workloads.batched_uneven(96) if 2 * math.pi * c.r2 / c.lam > 100][:6]
    assert len(cases) >= 3
    try:
        assert lib.lmieb_set_user_angle_part(64) == 0
        many = abi.solve_batch(lib, cases, n_threads=4)
        assert lib.lmieb_set_user_angle_part(4096) == 0
        one = abi.solve_batch(lib, cases, n_threads=4)
    finally:
        lib.lmieb_set_user_angle_part(256)
    for i, (a, b) in enumerate(zip(many, one)):
        assert a.rc == 0 and b.rc == 0 and a.n_coef == b.n_coef, i
        for name in ("pf", "pf_l"):
            assert libs.relmax(getattr(a, name), getattr(b, name)) <= 1e-13, (i, name)


def test_pipelined_calls_replay_their_parts_as_graphs():
    """A call cut into four parts hands each of the two slots two parts in
    turn; each slot keeps the graphs of its recent plans, so repeating the
    call replays every part (captured on the second call): the results are
    those of the first, kernel-by-kernel call bit for bit."""
    import ctypes as C
    lib = libs.product()
    lib.lmieb_graph_stats.argtypes = [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    def stats():
        a, b = C.c_longlong(), C.c_longlong()
        lib.lmieb_graph_stats(C.byref(a), C.byref(b))
        return a.value, b.value
    cases = workloads.batched_uneven(96)
    try:
        lib.lmieb_set_pipeline(4)
        first = abi.solve_batch(lib, cases, n_threads=4)
        c0, r0 = stats()
        for _ in range(3):
            again = abi.solve_batch(lib, cases, n_threads=4)
        c1, r1 = stats()
    finally:
        lib.lmieb_set_pipeline(0)
    assert c1 - c0 <= 4 and r1 - r0 >= 8, (c0, r0, c1, r1)
    for i, (a, b) in enumerate(zip(first, again)):
        assert a.rc == 0 and b.rc == 0 and a.n_coef == b.n_coef and a.scalars == b.scalars, i
        for name in ("gc", "pf", "gc_l", "pf_l"):
            assert np.array_equal(getattr(a, name), getattr(b, name)), (i, name)


def test_repeated_plan_is_replayed_as_a_graph():
    """A solve whose structure repeats (here the refractive index changes
    between calls, the radii, orders and angles do not) is captured the
    second time it comes to a slot (the library alternates two) and replayed
    from then on; the replayed results are the kernel-by-kernel ones bit for
    bit, and a changed structure goes back to launching kernel by kernel."""
    import ctypes as C
    lib = libs.product()
    lib.lmieb_graph_stats.argtypes = [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    def stats():
        a, b = C.c_longlong(), C.c_longlong()
        lib.lmieb_graph_stats(C.byref(a), C.byref(b))
        return a.value, b.value
    base = all_cases()["c2"]
    variants = [dataclasses.replace(base, mr=1.335 + 0.01 * i, mi=1e-6 * (1 + i)) for i in range(4)]
    # kernel by kernel: the first sight of each (a different structure in between)
    other = all_cases()["gamma"]
    first = []
    for v in variants:
        first.append(libs.run_product(v))
        libs.run_product(other)
    c0, r0 = stats()
    # the same structure call after call: captured once, then replayed
    again = [libs.run_product(v) for v in variants + variants]
    c1, r1 = stats()
    assert 1 <= c1 - c0 <= 2 and r1 - r0 >= 2 * len(variants) - 2, (c0, r0, c1, r1)
    for a, b in zip(first + first, again):
        assert a.n_coef == b.n_coef and a.scalars == b.scalars
        for name in ("gc", "pf", "gc_l", "pf_l"):
            assert np.array_equal(getattr(a, name), getattr(b, name)), name
    # another structure: launched kernel by kernel again
    libs.run_product(other)
    assert stats() == (c1, r1)
