"""Split-precision (3xTF32) angular contraction on the tensor cores.

lmie_solution_batch2(..., LMIEB_PRECISION_TF32X3) runs K3 through tcgen05.mma
with each operand split into two TF32 terms and FP32 accumulation;
everything else stays FP64 (and cases under 16 orders keep the FP64 K3).  The
FP64 form of the same library is the reference here: it is pinned to the
reference implementation at 1e-10 by the parity tests.

This form's contract is narrower than the int8 form's (test_oz_gpu.py, which
meets every bound on every case):
  - cross sections, g, reff/veff ...: not touched by K3, identical to FP64;
  - expansions (gc, lc, gc_l, lc_l) over the shorter n_coef: <= 1e-6 of each
    array's largest element;
  - the truncation n_coef is NOT the FP64 form's in general: it is the first
    l with |beta_l| <= accuracy, and the FP32-accumulated contraction leaves
    1e-6 .. 4e-5 of absolute noise on the tail beta_l while the FP64 tail
    passes the 1e-7 threshold within a few 1e-9 (measured over 256 seeded
    uneven cases: 119 kept the FP64 n_coef).  Where the truncations differ
    the user-angle phase matrix, summed from the kept coefficients, differs
    by the dropped or added terms (up to 3e-6 of pf's largest element and
    2.4e-4 of pf_l's): test_truncation_differences_are_bounded bounds it
    on every case rather than skipping those cases;
  - with accuracy 0 (no truncation) the phase matrix at the user angles
    carries only the contraction's error: <= 1e-6 on every case.
One named case is held to a looser bound on its linearised arrays: eight
radii at x ~ 1000 (x1000_few_radii), where no averaging over a size
distribution hides the operand split's ~22 bits in a derivative of a
normalised quadratic form: pf_l 2.0e-6, unchanged by shorter segments
(measured 2.3e-6 / 2.0e-6 / 3.4e-6 with segments of 1 / 2 / 4 chunks).
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
VALUE_TOL = 1e-6
DERIV_TOL = 1e-6


def _both(cases, n_threads=8):
    lib = libs.product()
    ref = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_FP64)
    got = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_TF32X3)
    return ref, got


def _check(got, want, label, deriv_tol=DERIV_TOL):
    assert got.rc == 0 and want.rc == 0, label
    err = libs.compare(got, want)
    scal = {k: v for k, v in err.items()
            if k not in libs.ARRAYS and k != "n_coef" and v > SCALARS_TOL}
    assert not scal, (label, scal)
    same_n = got.n_coef == want.n_coef
    for name in ("gc", "lc") + (("pf",) if same_n else ()):
        if name in err:
            assert err[name] <= VALUE_TOL, (label, name, err[name])
    for name in ("gc_l", "lc_l") + (("pf_l",) if same_n else ()):
        if name in err:
            assert err[name] <= deriv_tol, (label, name, err[name])
    return err


@pytest.mark.parametrize("K", [16, 64, 256])
def test_selftest_contraction(K):
    """One 128 x 128 product through the same operand split, layout,
    descriptors and tensor-memory reads, against FP64 on the host; a single
    FP32 accumulation over K, so the bound grows with K."""
    e = C.c_double(-1.)
    assert libs.product().lmieb_tc_selftest(K, C.byref(e)) == 0
    assert 0. <= e.value < 2e-8 * K + 5e-7, e.value


def test_selftest_rejects_bad_k():
    e = C.c_double(-1.)
    assert libs.product().lmieb_tc_selftest(24, C.byref(e)) == -1


@pytest.mark.parametrize("name, deriv_tol", [("c1", DERIV_TOL), ("c2", DERIV_TOL), ("example", DERIV_TOL),
                                             ("x1000_few_radii", 3e-6)])
def test_named_cases(name, deriv_tol):
    (ref,), (got,) = _both([all_cases()[name]])
    _check(got, ref, name, deriv_tol)


def test_uneven_batch():
    """A slice of the seeded uneven workload (size parameters up to ~1000,
    derivatives of mr, mi, r_eff, v_eff): the bounds above on every case
    whose truncation agrees with FP64."""
    cases = workloads.batched_uneven(192)
    ref, got = _both(cases, n_threads=16)
    for i, (g, r) in enumerate(zip(got, ref)):
        _check(g, r, f"case {i}")


def test_truncation_differences_are_bounded():
    """Every case of the slice, including those whose truncation differs: the
    user-angle phase matrix within 1e-5 of its largest element and its
    linearisations within 5e-3 -- the dropped or added tail terms (measured
    on this slice: 3.0e-6 and 2.4e-4), which is why this form does not meet
    the 1e-6 target and the int8 form does."""
    cases = workloads.batched_uneven(192)
    ref, got = _both(cases, n_threads=16)
    differ = 0
    for i, (g, r) in enumerate(zip(got, ref)):
        assert g.rc == 0 and r.rc == 0, i
        differ += g.n_coef != r.n_coef
        assert libs.relmax(g.pf, r.pf) <= 1e-5, (i, libs.relmax(g.pf, r.pf))
        assert libs.relmax(g.pf_l, r.pf_l) <= 5e-3, (i, libs.relmax(g.pf_l, r.pf_l))
    assert 0 < differ < len(cases), differ


def test_pf_with_untruncated_expansion():
    """With accuracy 0 nothing is truncated, so the user-angle phase matrix
    carries only the contraction's error."""
    cases = [dataclasses.replace(c, accuracy=0.) for c in workloads.batched_uneven(48)]
    ref, got = _both(cases, n_threads=16)
    for i, (g, r) in enumerate(zip(got, ref)):
        assert g.n_coef == r.n_coef, i
        err = _check(g, r, f"case {i}")
        assert err["pf"] <= VALUE_TOL, (i, err["pf"])


def test_without_derivatives_and_legendre():
    """nd = 0 (two operand rows per radius) and the Legendre expansion path."""
    base = all_cases()["c2"]
    cases = []
    for lc in (0, 1):
        cases.append(dataclasses.replace(base, derivs=[], calc_lc=lc, calc_gc=1 - lc))
    ref, got = _both(cases)
    for i, (g, r) in enumerate(zip(got, ref)):
        _check(g, r, f"variant {i}")


def test_split_mode_is_deterministic():
    cases = workloads.batched_uneven(32)
    lib = libs.product()
    a = abi.solve_batch(lib, cases, n_threads=8, precision=abi.PRECISION_TF32X3)
    b = abi.solve_batch(lib, cases, n_threads=8, precision=abi.PRECISION_TF32X3)
    for x, y in zip(a, b):
        assert np.array_equal(x.pf, y.pf) and np.array_equal(x.gc, y.gc)


def test_small_particles_keep_the_fp64_angular_stage():
    """Cases under 16 orders (size parameter below ~2.5) run the FP64 K3 in a
    split-precision batch, mixed with tensor-core cases: their results are the
    FP64 form's to round-off."""
    tiny = [dataclasses.replace(c, r2=c.lam * 0.35, r1=c.lam * 0.001) for c in workloads.batched_uneven(6)]
    cases = tiny[:3] + workloads.batched_uneven(12)[6:] + tiny[3:]
    ref, got = _both(cases, n_threads=8)
    for i in list(range(3)) + list(range(len(cases) - 3, len(cases))):
        err = libs.compare(got[i], ref[i])
        assert got[i].n_coef == ref[i].n_coef, i
        assert not {k: v for k, v in err.items() if v > 1e-12}, (i, err)
    for i in range(3, len(cases) - 3):
        _check(got[i], ref[i], f"case {i}")


def test_precision_stress_large_particles():
    """Size parameter 5000 (n1 = 5077, 10154 Gauss angles, 8000 radii, four
    derivatives): every output array within 1e-6 of the FP64 form."""
    cases = workloads.precision_stress(2)
    ref, got = _both(cases, n_threads=16)
    for i, (g, r) in enumerate(zip(got, ref)):
        assert g.n_coef == r.n_coef, i
        _check(g, r, f"case {i}")
