"""Fixed-point angular contraction on the int8 tensor cores
(lmie_solution_batch2(..., LMIEB_PRECISION_INT8)).

Every operand value is scaled by powers of two and split into six signed
8-bit digits whose products are summed exactly in int32 (tcgen05.mma
kind::i8); everything else is the FP64 form's arithmetic.  The FP64 form of
the same library is the reference here: it is pinned to the reference
implementation at 1e-10 by the parity tests.  The contract checked below:
  - the truncation n_coef is the FP64 form's in every case: cases whose
    |beta_l| come within the contraction's error band of `accuracy` are
    solved again in FP64 within the same call;
  - cross sections, g, reff/veff ...: identical to FP64 (not touched);
  - every output array (gc, lc, pf and their derivatives) within 1e-9 of FP64
    as max|got - want| / max|want|, and every derivative slice (one
    derivative, one element) within 1e-8 of its own maximum -- the split-
    precision target is 1e-6, so these bounds leave three orders of margin
    over what the contraction carries (measured: 6e-12 per array, 2e-10 per
    slice over the 4096-case uneven workload).
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import libs
from cases import all_cases
from lmie_b200 import abi, workloads

pytestmark = pytest.mark.gpu

SCALARS_TOL = 1e-13
ARRAY_TOL = 1e-9
SLICE_TOL = 1e-8


def band(n1max):
    """The re-solve band of a case whose radii reach n1max orders (oz_layout.cuh
    oz_trunc_band): |beta_l(int8) - beta_l(FP64)| <= band (2l + 1) near the
    truncation threshold."""
    return 2.5e-13 if n1max <= 1152 else 5e-12


def n1(x):
    """The reference's truncation n1 of size parameter x (src/lmie_core.c:18-38)."""
    return int(x + 4.05 * x ** (1. / 3.) + 2.)


def tail_error(g, r):
    """max |beta_l(got) - beta_l(want)| / (2l + 1) over the l whose FP64
    |beta_l| lies within 1e-9 .. 1e-5 of 2l + 1, around the threshold 1e-7."""
    b = r.gc[0]
    ell = np.arange(b.shape[0])
    m = (np.abs(b) <= 1e-5 * (2 * ell + 1)) & (np.abs(b) >= 1e-9 * (2 * ell + 1))
    return float(np.max(np.abs(g.gc[0] - b)[m] / (2 * ell[m] + 1))) if m.any() else 0.


def _lib():
    lib = libs.product()
    lib.lmieb_last_redo.restype = C.c_int
    lib.lmieb_last_redo.argtypes = [C.POINTER(C.c_longlong)]
    lib.lmieb_oz_selftest.restype = C.c_int
    lib.lmieb_oz_selftest.argtypes = [C.c_int, C.POINTER(C.c_double)]
    return lib


def _redo(lib):
    n = C.c_longlong(-1)
    assert lib.lmieb_last_redo(C.byref(n)) == 0
    return n.value


def _both(cases, n_threads=16):
    lib = _lib()
    ref = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_FP64)
    got = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_INT8)
    return ref, got, _redo(lib)


def _slices(a, b):
    worst = 0.0
    for i in range(b.shape[0]):
        for e in range(b.shape[1]):
            m = float(np.max(np.abs(b[i, e])))
            if m > 0:
                worst = max(worst, float(np.max(np.abs(a[i, e] - b[i, e]))) / m)
    return worst


def _check(got, want, label):
    assert got.rc == 0 and want.rc == 0, label
    assert got.n_coef == want.n_coef, (label, got.n_coef, want.n_coef)
    err = libs.compare(got, want)
    scal = {k: v for k, v in err.items() if k not in libs.ARRAYS and k != "n_coef" and v > SCALARS_TOL}
    assert not scal, (label, scal)
    for name in ("gc", "lc", "pf", "gc_l", "lc_l", "pf_l"):
        if name in err:
            assert err[name] <= ARRAY_TOL, (label, name, err[name])
    for name in ("gc_l", "lc_l", "pf_l"):
        a, b = getattr(got, name), getattr(want, name)
        if b is not None:
            s = _slices(a, b)
            assert s <= SLICE_TOL, (label, name, s)
    return err


@pytest.mark.parametrize("K", [32, 256, 5120])
def test_selftest_contraction(K):
    """One 128 x 64 product through the same scaling, digit slices, tensor
    memory, products and exact combination, against long-double sums: the
    error of each element relative to max|a_i.| max|b_n.|."""
    e = C.c_double(-1.)
    assert _lib().lmieb_oz_selftest(K, C.byref(e)) == 0
    assert 0. <= e.value < 1e-11, e.value


def test_selftest_rejects_bad_k():
    e = C.c_double(-1.)
    assert _lib().lmieb_oz_selftest(48, C.byref(e)) == -1
    assert _lib().lmieb_oz_selftest(32 * 161, C.byref(e)) == -1


@pytest.mark.parametrize("name", ["c1", "c2", "example", "x1000_few_radii", "nine_derivs", "lognormal_gc_lc"])
def test_named_cases(name):
    (ref,), (got,), _ = _both([all_cases()[name]])
    _check(got, ref, name)


def test_uneven_workload_every_case():
    """The whole 4096-case uneven workload (size parameters up to ~1000,
    derivatives of mr, mi, r_eff, v_eff): the same n_coef in every case and
    every array and derivative slice within the bounds."""
    cases = workloads.batched_uneven(4096)
    ref, got, redo = _both(cases)
    for i, (g, r) in enumerate(zip(got, ref)):
        _check(g, r, f"case {i}")
    # the re-solve is rare: the band is a few 1e-13 (2l + 1) wide
    assert 0 <= redo < len(cases) // 50, redo


def test_expansion_error_within_the_band():
    """With accuracy 0 nothing is truncated: the expansion coefficients near
    the threshold of 1024 uneven cases and of the large-particle
    configuration against FP64, the bound the re-solve band relies on, with a
    factor of 1.5 to spare."""
    import math
    cases = [dataclasses.replace(c, accuracy=0.) for c in workloads.batched_uneven(1024)]
    cases += [dataclasses.replace(c, accuracy=0.) for c in workloads.precision_stress(2)]
    ref, got, redo = _both(cases)
    assert redo == 0
    for i, (c, g, r) in enumerate(zip(cases, got, ref)):
        assert g.n_coef == r.n_coef
        e = tail_error(g, r)
        assert e <= band(n1(2 * math.pi * c.r2 / c.lam)) / 1.5, (i, e)


def test_truncation_at_the_threshold_is_solved_in_fp64():
    """A case whose accuracy is set to one of its own |beta_l|: the truncation
    sits exactly at the threshold, the case is solved again in FP64, and its
    outputs are the FP64 form's bit for bit."""
    base = all_cases()["c2"]
    lib = _lib()
    (full,) = abi.solve_batch(lib, [dataclasses.replace(base, accuracy=0.)], precision=abi.PRECISION_FP64)
    beta = np.abs(full.gc[0])
    # the first |beta_l| <= 1e-7: every earlier one is larger, so an accuracy
    # equal to it puts the truncation exactly on the threshold
    l0 = int(np.argmax(beta <= 1e-7))
    assert l0 > 0 and beta[l0] > 0
    case = dataclasses.replace(base, accuracy=float(beta[l0]))
    (ref,), (got,), redo = _both([case])
    assert redo == 1
    assert got.n_coef == ref.n_coef
    for name in ("gc", "pf", "gc_l", "pf_l"):
        assert np.array_equal(getattr(got, name), getattr(ref, name)), name


def test_re_solves_in_every_part_are_the_fp64_form():
    """Cases on the truncation threshold in each of four pipelined parts: their
    FP64 re-solves copy the coefficients from the int8 part's device memory
    while later parts reuse the same buffers; every re-solved case is the FP64
    form's bit for bit and the others stay within the bounds."""
    import math
    lib = _lib()
    cases, at = [], []
    for i, c in enumerate(workloads.batched_uneven(48)):
        # (cases under 16 orders keep the FP64 angular stage: no re-solve)
        if i % 3 == 0 and n1(2 * math.pi * c.r2 / c.lam) >= 16:
            (full,) = abi.solve_batch(lib, [dataclasses.replace(c, accuracy=0.)], precision=abi.PRECISION_FP64)
            beta = np.abs(full.gc[0])
            l0 = int(np.argmax(beta <= 1e-7))
            if l0 > 0 and beta[l0] > 0:
                c = dataclasses.replace(c, accuracy=float(beta[l0]))
                at.append(i)
        cases.append(c)
    assert len(at) >= 4, at
    lib.lmieb_set_pipeline.argtypes = [C.c_int]
    lib.lmieb_set_pipeline(4)
    try:
        ref, got, redo = _both(cases)
    finally:
        lib.lmieb_set_pipeline(0)
    assert redo >= len(at), (redo, at)
    for i, (g, r) in enumerate(zip(got, ref)):
        if i in at:
            assert g.n_coef == r.n_coef, i
            for name in ("gc", "pf", "gc_l", "pf_l"):
                assert np.array_equal(getattr(g, name), getattr(r, name)), (i, name)
        else:
            _check(g, r, f"case {i}")


def test_precision_stress_large_particles():
    """Size parameter 5000 (n1 = 5077, 10154 Gauss angles, 8000 radii, four
    derivatives): 159 chunks per radius group, near the exact-sum limit."""
    cases = workloads.precision_stress(2)
    ref, got, _ = _both(cases)
    for i, (g, r) in enumerate(zip(got, ref)):
        _check(g, r, f"case {i}")


def test_small_particles_keep_the_fp64_angular_stage():
    """Cases under 16 orders run the FP64 K3 in an int8 batch, mixed with
    tensor-core cases: their results are the FP64 form's to round-off."""
    tiny = [dataclasses.replace(c, r2=c.lam * 0.35, r1=c.lam * 0.001) for c in workloads.batched_uneven(6)]
    cases = tiny[:3] + workloads.batched_uneven(12)[6:] + tiny[3:]
    ref, got, _ = _both(cases)
    for i in list(range(3)) + list(range(len(cases) - 3, len(cases))):
        err = libs.compare(got[i], ref[i])
        assert got[i].n_coef == ref[i].n_coef, i
        assert not {k: v for k, v in err.items() if v > 1e-12}, (i, err)
    for i in range(3, len(cases) - 3):
        _check(got[i], ref[i], f"case {i}")


def test_int8_mode_is_deterministic():
    cases = workloads.batched_uneven(64)
    lib = _lib()
    a = abi.solve_batch(lib, cases, n_threads=8, precision=abi.PRECISION_INT8)
    b = abi.solve_batch(lib, cases, n_threads=8, precision=abi.PRECISION_INT8)
    for x, y in zip(a, b):
        assert np.array_equal(x.pf, y.pf) and np.array_equal(x.gc, y.gc) and np.array_equal(x.gc_l, y.gc_l)


def test_without_derivatives_and_legendre():
    """nd = 0 (two operand rows per radius, 16 radii per group) and the
    Legendre expansion path."""
    base = all_cases()["c2"]
    cases = [dataclasses.replace(base, derivs=[], calc_lc=lc, calc_gc=1 - lc) for lc in (0, 1)]
    ref, got, _ = _both(cases)
    for i, (g, r) in enumerate(zip(got, ref)):
        _check(g, r, f"variant {i}")
