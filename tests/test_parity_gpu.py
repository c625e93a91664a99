"""Parity of the CUDA solve with the reference, through the C ABI.

Every output array of lmie_solution is compared with the reference's own
output (golden fixtures made from the reference library, and the reference
library itself when it is present) by the max-norm relative error
max|got - want| / max|want|.  The plain FP64 path must agree to 1e-10 on
every output; n_coef may differ by one when a coefficient sits at the
truncation threshold (then the shorter length is compared).
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import libs
from cases import all_cases, c2_case, example_case
from lmie_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _assert_parity(got, want, tol=TOL, label=""):
    assert got.rc == 0, label
    err = libs.compare(got, want)
    assert err["n_coef"] <= 1, (label, got.n_coef, want.n_coef)
    bad = {k: v for k, v in err.items() if k != "n_coef" and v > tol}
    assert not bad, (label, bad)


@pytest.mark.parametrize("name", list(all_cases().keys()))
def test_parity_with_reference_fixture(name):
    case = all_cases()[name]
    want = libs.golden(name)
    assert want is not None
    _assert_parity(libs.run_product(case), want, label=name)


@pytest.mark.parametrize("name", ["c1", "gamma", "nine_derivs", "lognormal_gc_lc", "mono"])
def test_parity_with_oracle(name):
    case = all_cases()[name]
    _assert_parity(libs.run_product(case), libs.run_oracle(case), label=name)


@pytest.mark.skipif(libs.reference() is None, reason="reference library not built here")
def test_parity_with_live_reference_threads():
    """Against the reference run with its own thread pool (different radius
    summation order), on the reference's example."""
    case = example_case()
    _assert_parity(libs.run_product(case), libs.run_reference(case, 4), label="example")


def test_example_out_golden():
    """The reference's printed golden output (7 digits)."""
    with np.load(libs.GOLDEN / "example_out.npz") as z:
        scal, names, gc, pf = z["scalars"], list(z["scalar_names"]), z["gc"], z["pf"]
    got = libs.run_product(example_case())
    assert got.n_coef == 246
    for i, k in enumerate(names):
        assert abs(got.scalars[k] - scal[0, i]) <= 1.5e-6 * abs(scal[0, i])
    tab = lambda a, b: np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-12 * np.max(np.abs(b)))
    assert tab(got.gc, gc[0]) and tab(got.pf, pf[0])
    for d in range(4):
        assert tab(got.gc_l[d], gc[1 + d]) and tab(got.pf_l[d], pf[1 + d])


def test_bitwise_reproducible():
    """Fixed-order reductions: the same input gives the same bits."""
    a = libs.run_product(c2_case())
    b = libs.run_product(c2_case())
    for name in ("gc", "pf", "gc_l", "pf_l"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert a.scalars == b.scalars


def test_solution2_without_derivatives():
    """lmie_solution2 (no derivative arguments) gives the value outputs of
    lmie_solution."""
    case = all_cases()["gamma"]
    full = libs.run_product(case)
    lib = libs.product()
    mc = lib.lmie_calc_max_coef(case.lam, abi.SIZE_DIST["gamma"], case.a1, case.a2, case.a3,
                                case.r1, case.r2)
    gc = abi.lmie_out_data()  # just for the row-pointer allocators
    s = abi.lmie_in_data()
    s.calc_gc, s.calc_lc, s.calc_pf, s.n_angles, s.n_derivs = 1, 0, 1, case.n_angles, 0
    lib.lmie_out_alloc.argtypes = [C.POINTER(abi.lmie_in_data), C.POINTER(abi.lmie_out_data), C.c_int]
    lib.lmie_out_alloc(C.byref(s), C.byref(gc), mc)
    d = C.c_double
    vals = [d() for _ in range(15)]
    n_coef = C.c_int()
    sv1 = abi.PPD()
    sv2 = abi.PPPD()
    lib.lmie_solution2.restype = C.c_int
    rc = lib.lmie_solution2(1, 0, 1, abi.SIZE_DIST["gamma"], case.n_int1, case.n_int2, case.n_quad,
                            case.n_angles, 0, d(case.lam), d(case.mr), d(case.mi), d(case.a1),
                            d(case.a2), d(case.a3), d(case.a4), d(case.a5), d(case.r1), d(case.r2),
                            d(case.accuracy), C.byref(n_coef), *[C.byref(v) for v in vals[:13]],
                            gc.gc, None, gc.theta, gc.pf, C.byref(sv1), C.byref(sv2), 0, 1, 0)
    assert rc == 0
    assert n_coef.value == full.n_coef
    names = ["r1", "r2", "norm", "reff", "veff", "gavg", "vavg", "ravg", "rvw", "cext", "csca",
             "cbak", "g"]
    # value outputs of a solve without derivatives agree with those of a
    # solve with derivatives to the last few bits (the two runs use different
    # kernel instantiations, which may contract FMAs differently)
    for v, k in zip(vals[:13], names):
        assert libs.rel_scalar(v.value, full.scalars[k]) < 1e-14, k
    got_gc = np.ctypeslib.as_array(gc.gc[0], shape=(6, mc))[:, :full.n_coef]
    assert libs.relmax(got_gc, full.gc) < 1e-14
    lib.lmie_out_free(C.byref(gc), 0)


def test_fortran_shim_column_major():
    """lmie_solution2_l_ (the F77/F90 entry) on flat column-major arrays:
    gc(max_coef,6), gc_l(max_coef,6,nd), pf(n_angles,6), pf_l(n_angles,6,nd)."""
    case = all_cases()["gamma"]
    case = dataclasses.replace(case, derivs=abi.deriv_unit("mr", "a1", "r2"))
    full = libs.run_product(case)
    lib = libs.product()
    nd, na = case.n_derivs, case.n_angles
    mc = lib.lmie_calc_max_coef(case.lam, abi.SIZE_DIST["gamma"], case.a1, case.a2, case.a3,
                                case.r1, case.r2)
    blk = abi.InputBlock(case)
    D = lambda v: C.byref(C.c_double(v))
    I = lambda v: C.byref(C.c_int(v))
    arr = lambda n: np.zeros(n, dtype=np.float64)
    gc, gcl = arr(6 * mc), arr(6 * mc * nd)
    pf, pfl, theta = arr(6 * na), arr(6 * na * nd), arr(na)
    sc = [arr(1) for _ in range(13)]
    scl = [arr(nd) for _ in range(13)]
    p = lambda a: a.ctypes.data_as(abi.PD)
    n_coef = C.c_int()
    sv1, sv2 = abi.PPD(), abi.PPPD()
    dt = C.c_int(abi.SIZE_DIST["gamma"])
    lib.lmie_solution2_l_.restype = C.c_int
    rc = lib.lmie_solution2_l_(I(1), I(0), I(1), C.byref(dt), I(case.n_int1), I(case.n_int2),
                               I(case.n_quad), I(na), I(nd), I(0), D(case.lam), D(case.mr), D(case.mi),
                               D(case.a1), D(case.a2), D(case.a3), D(case.a4), D(case.a5), D(case.r1),
                               D(case.r2), *[p(blk.arrays[n]) for n in abi.DERIV_INPUTS],
                               D(case.accuracy), C.byref(n_coef), *[p(a) for a in sc],
                               p(gc), None, p(theta), p(pf), *[p(a) for a in scl],
                               p(gcl), None, p(pfl), C.byref(sv1), C.byref(sv2), I(mc), I(0), I(1),
                               I(0))
    assert rc == 0 and n_coef.value == full.n_coef
    nc = full.n_coef
    assert np.array_equal(gc.reshape(6, mc)[:, :nc], full.gc)
    assert np.array_equal(gcl.reshape(nd, 6, mc)[:, :, :nc], full.gc_l)
    assert np.array_equal(pf.reshape(6, na), full.pf)
    assert np.array_equal(pfl.reshape(nd, 6, na), full.pf_l)
    assert sc[9][0] == full.scalars["cext"] and np.array_equal(scl[10], full.scalars_l["csca"])


def test_save_control_reweighting():
    """save_control 1 stores per-radius kernels; save_control 2 re-weights
    them for a new distribution shape without Mie work (reference
    src/lmie_schedule.c:1078-1124).  Checked against the oracle."""
    case = all_cases()["save1"]
    got = libs.run_product(case)
    want = libs.golden("save1")
    _assert_parity(got, want, label="save1")
    # re-weight for a new effective variance through both libraries
    new = dataclasses.replace(case, a2=0.25, save_control=2)
    results = []
    for lib, kind in ((libs.product(), "lmie"), (libs.oracle(), "oracle")):
        blk = abi.InputBlock(new)
        out = abi.lmie_out_data()
        s1 = np.ascontiguousarray(want.save1)
        s2 = np.ascontiguousarray(want.save2)
        n, nq = s2.shape[1], s2.shape[2]
        rows1 = (abi.PD * 4)(*[s1[e].ctypes.data_as(abi.PD) for e in range(4)])
        rows2 = [(abi.PD * n)(*[s2[e, r].ctypes.data_as(abi.PD) for r in range(n)]) for e in range(4)]
        rows2p = (abi.PPD * 4)(*[C.cast(r, abi.PPD) for r in rows2])
        out.save1 = C.cast(rows1, abi.PPD)
        out.save2 = C.cast(rows2p, abi.PPPD)
        if kind == "oracle":
            mc = lib.oracle_calc_max_coef(new.lam, 4, new.a1, new.a2, 0.0, new.r1, new.r2)
            lib_out_alloc = None
            rc = _oracle_solve_prealloc(lib, blk, out, mc, new)
        else:
            mc = lib.lmie_calc_max_coef(new.lam, 4, new.a1, new.a2, 0.0, new.r1, new.r2)
            rc = lib.lmie_solution(C.byref(blk.s), C.byref(out), 1, 0, 1, 0)
        assert rc == 0
        results.append(abi.read_output(new, out, mc))
    _assert_parity(results[0], results[1], label="save_control 2")


def _oracle_solve_prealloc(lib, blk, out, mc, case):
    return lib.oracle_solution(C.byref(blk.s), C.byref(out), 1)


def _reweight(lib, kind, case, s1, s2):
    """A save_control 2 solve of `case` on the kernels s1 [4, n], s2 [4, n, nq]
    (numpy), handed over through row pointers as LMie callers do."""
    blk = abi.InputBlock(case)
    out = abi.lmie_out_data()
    s1 = np.ascontiguousarray(s1)
    s2 = np.ascontiguousarray(s2)
    n = s2.shape[1]
    rows1 = (abi.PD * 4)(*[s1[e].ctypes.data_as(abi.PD) for e in range(4)])
    rows2 = [(abi.PD * n)(*[s2[e, r].ctypes.data_as(abi.PD) for r in range(n)]) for e in range(4)]
    rows2p = (abi.PPD * 4)(*[C.cast(r, abi.PPD) for r in rows2])
    out.save1 = C.cast(rows1, abi.PPD)
    out.save2 = C.cast(rows2p, abi.PPPD)
    if kind == "oracle":
        mc = lib.oracle_calc_max_coef(case.lam, 4, case.a1, case.a2, 0.0, case.r1, case.r2)
        rc = lib.oracle_solution(C.byref(blk.s), C.byref(out), 1)
    else:
        mc = lib.lmie_calc_max_coef(case.lam, 4, case.a1, case.a2, 0.0, case.r1, case.r2)
        rc = lib.lmie_solution(C.byref(blk.s), C.byref(out), 1, 0, 1, 0)
    assert rc == 0
    return abi.read_output(case, out, mc)


def _save_stats(lib):
    h, m = C.c_longlong(), C.c_longlong()
    lib.lmieb_save_cache_stats(C.byref(h), C.byref(m))
    return h.value, m.value


def test_save_control_kernels_stay_on_the_device():
    """After a save_control 1 solve its kernels stay on the device: a
    save_control 2 call given the same values (hashed through its row
    pointers) uploads nothing; changed values are uploaded and kept in their
    turn.  Every result against the oracle on the same kernels."""
    lib, orc = libs.product(), libs.oracle()
    case = all_cases()["save1"]
    first = libs.run_product(case)
    assert first.rc == 0
    s1, s2 = first.save1, first.save2
    new = dataclasses.replace(case, a2=0.25, save_control=2)
    h0, m0 = _save_stats(lib)
    got = _reweight(lib, "lmie", new, s1, s2)
    assert _save_stats(lib) == (h0 + 1, m0)
    _assert_parity(got, _reweight(orc, "oracle", new, s1, s2), label="kept kernels")
    # changed kernels: uploaded, then kept
    s2b = s2.copy()
    s2b[1, 3, :] *= 1.5
    got2 = _reweight(lib, "lmie", new, s1, s2b)
    assert _save_stats(lib) == (h0 + 1, m0 + 1)
    _assert_parity(got2, _reweight(orc, "oracle", new, s1, s2b), label="changed kernels")
    assert not np.array_equal(got2.pf, got.pf)
    new3 = dataclasses.replace(new, a2=0.3)
    got3 = _reweight(lib, "lmie", new3, s1, s2b)
    assert _save_stats(lib) == (h0 + 2, m0 + 1)
    _assert_parity(got3, _reweight(orc, "oracle", new3, s1, s2b), label="kept changed kernels")


def test_invalid_inputs_return_minus_one():
    lib = libs.product()
    assert abi.solve(lib, abi.Case(calc_gc=0, calc_lc=0, calc_pf=1)).rc == -1
    assert abi.solve(lib, abi.Case(dist=0)).rc == -1          # SIZE_DIST_NONE
    assert abi.solve(lib, abi.Case(n_quad=0)).rc == -1        # no radii
    assert abi.solve(lib, abi.Case(save_control=5)).rc == -1
    # and the library keeps working afterwards
    assert abi.solve(lib, abi.Case()).rc == 0


def test_derivatives_against_central_differences():
    """Forward-linearized outputs vs central finite differences of the CUDA
    solve itself (step 1e-6 relative), on a reduced cloud-droplet case."""
    base = abi.Case(dist="gamma", lam=0.865, mr=1.335, mi=1e-3, a1=2.0, a2=0.1, r1=0.01, r2=8.0,
                    n_int2=2, n_quad=100, accuracy=0.0,
                    derivs=abi.deriv_unit("mr", "mi", "a1", "a2"))
    got = libs.run_product(base)
    assert got.rc == 0
    params = {"mr": "mr", "mi": "mi", "a1": "a1", "a2": "a2"}
    for d, (p, field) in enumerate(params.items()):
        v = getattr(base, field)
        h = 1e-6 * abs(v)
        up = libs.run_product(dataclasses.replace(base, derivs=[], **{field: v + h}))
        dn = libs.run_product(dataclasses.replace(base, derivs=[], **{field: v - h}))
        for k in ("cext", "csca", "cbak", "g"):
            fd = (up.scalars[k] - dn.scalars[k]) / (2 * h)
            an = got.scalars_l[k][d]
            assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3 * abs(got.scalars[k])), (p, k, fd, an)
        fd = (up.pf - dn.pf) / (2 * h)
        assert libs.relmax(got.pf_l[d], fd) < 1e-4, p
        nc = min(up.n_coef, dn.n_coef, got.n_coef)
        fd = (up.gc[:, :nc] - dn.gc[:, :nc]) / (2 * h)
        assert libs.relmax(got.gc_l[d][:, 1:nc], fd[:, 1:]) < 1e-4, p


def test_save_control_without_angular_outputs():
    """save_control 1 and 2 with no expansion or phase matrix requested (only
    the per-radius cross sections are saved): the kept kernels are save1
    alone, and the re-weighted cross sections match the oracle."""
    lib, orc = libs.product(), libs.oracle()
    case = dataclasses.replace(all_cases()["save1"], calc_gc=0, calc_lc=0, calc_pf=0)
    first = libs.run_product(case)
    assert first.rc == 0
    want_first = libs.run_oracle(case)
    _assert_parity(first, want_first, label="save_control 1 without angles")
    s1 = first.save1
    s2 = np.zeros((4, s1.shape[1], 1))
    new = dataclasses.replace(case, a2=0.25, save_control=2)
    h0, m0 = _save_stats(lib)
    got = _reweight(lib, "lmie", new, s1, s2)
    assert _save_stats(lib) == (h0 + 1, m0)
    _assert_parity(got, _reweight(orc, "oracle", new, s1, s2), label="re-weighted without angles")
