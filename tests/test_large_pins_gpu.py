"""The benchmark's sizes pinned to the reference itself: the large-particle
configuration with every output (size parameter up to 5000, n_coef 10156,
four derivatives) and eight cases of the 4096-case uneven workload with
size parameters from 502 to 1063 (tests/cases.py large_cases(); fixtures
made from the reference library by tests/golden/make_golden.py).

FP64, through lmie_solution and through the batch call: every output within
1e-10 of the reference as max|got - want| / max|want| (n_coef may differ by
one where a coefficient sits at the truncation threshold).  The int8
fixed-point batch form (within 1e-9 of the FP64 form by its contract): every
output array within 2e-9 of the reference, the scalars within 1e-10.
"""
import numpy as np
import pytest

import libs
from cases import large_cases
from lmie_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10
INT8_ARRAY_TOL = 2e-9


def _assert_parity(got, want, tol=TOL, array_tol=TOL, label=""):
    assert got.rc == 0, label
    err = libs.compare(got, want)
    assert err["n_coef"] <= 1, (label, got.n_coef, want.n_coef)
    bad = {k: v for k, v in err.items()
           if k != "n_coef" and v > (array_tol if k in libs.ARRAYS else tol)}
    assert not bad, (label, bad)


@pytest.mark.parametrize("name", list(large_cases()))
def test_solution_matches_reference(name):
    _assert_parity(libs.run_product(large_cases()[name]), libs.golden(name), label=name)


def _batch(precision):
    cases = large_cases()
    res = abi.solve_batch(libs.product(), list(cases.values()), n_threads=8, precision=precision)
    return [(name, got, libs.golden(name)) for name, got in zip(cases, res)]


def test_batch_fp64_matches_reference():
    for name, got, want in _batch(abi.PRECISION_FP64):
        _assert_parity(got, want, label=name)


def test_batch_int8_matches_reference():
    for name, got, want in _batch(abi.PRECISION_INT8):
        _assert_parity(got, want, array_tol=INT8_ARRAY_TOL, label=name)


def test_large_fixture_reaches_the_sizes():
    """The fixtures hold what they claim: n_coef ~ 2 x_max and every array."""
    want = libs.golden("x5000_full")
    assert want.n_coef > 10000 and want.gc_l.shape == (4, 6, want.n_coef) and want.pf_l.shape[0] == 4
    for name in large_cases():
        if name.startswith("uneven_"):
            w = libs.golden(name)
            assert w.n_coef > 1000 and w.pf_l is not None and np.all(np.isfinite(w.pf_l)), name
