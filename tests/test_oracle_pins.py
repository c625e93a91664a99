"""The CPU oracle is pinned to the reference before it is trusted.

(a) examples/example.out, the reference's golden output, at its 7 printed
    significant digits (tests/golden/example_out.npz);
(b) full-precision outputs of the reference library compiled from its own
    sources (tests/golden/ref_*.npz, made by tests/golden/make_golden.py);
(c) the reference library itself when it is present (oracle/_ref).
"""
import numpy as np
import pytest

import libs
from cases import all_cases, example_case, small_cases

# The oracle restates the reference's arithmetic in the same order, so it
# agrees with the single-threaded reference to a few ulps; 1e-12 leaves room
# for libm differences between machines.
TOL = 1e-12


def _check(got, want, tol):
    err = libs.compare(got, want)
    bad = {k: v for k, v in err.items() if v > tol}
    assert got.n_coef == want.n_coef
    assert not bad, bad


@pytest.mark.parametrize("name", list(small_cases().keys()) + ["example", "c2",
                                                              "large_x_cross_sections"])
def test_oracle_matches_reference_fixtures(name):
    case = all_cases()[name]
    want = libs.golden(name)
    assert want is not None, f"missing fixture ref_{name}.npz"
    got = libs.run_oracle(case)
    assert got.rc == 0
    _check(got, want, TOL)


@pytest.mark.parametrize("name", ["x5000_full", "uneven_2963"])
def test_oracle_matches_reference_at_large_size(name):
    """Size parameters 5000 (n_coef 10156, every output) and 1063 (2200
    radii of the uneven workload): a few seconds of oracle time each."""
    from cases import large_cases
    got = libs.run_oracle(large_cases()[name])
    assert got.rc == 0
    _check(got, libs.golden(name), TOL)


def test_oracle_matches_example_out():
    """7 significant digits of examples/example.out (value and the 4
    derivatives: mr, mi, a1, a2)."""
    with np.load(libs.GOLDEN / "example_out.npz") as z:
        scal = z["scalars"]
        names = list(z["scalar_names"])
        gc = z["gc"]
        pf = z["pf"]
        theta = z["theta"]
        n_coef = int(z["n_coef"])
    got = libs.run_oracle(example_case())
    assert got.n_coef == n_coef
    # printed with %14E: 7 significant digits -> relative 5e-7 of each value,
    # plus one unit in the last digit for values the reference's own rebuild
    # reproduces only to the 7th digit
    def close(a, b):
        return np.all(np.abs(a - b) <= 1.5e-6 * np.abs(b) + 1e-300)
    for i, k in enumerate(names):
        assert close(got.scalars[k], scal[0, i]), k
        for d in range(4):
            v = got.scalars_l[k][d]
            assert abs(v - scal[1 + d, i]) <= 1.5e-6 * abs(scal[1 + d, i]) + 1e-12, (k, d)
    np.testing.assert_allclose(got.theta, theta, rtol=0, atol=1e-5)
    # tables: compare relative to each table's scale (small entries are printed
    # with 7 digits of their own magnitude, so allow 1 unit in the 7th digit)
    def table_ok(a, b):
        return np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-12 * np.max(np.abs(b)))
    assert table_ok(got.gc, gc[0])
    assert table_ok(got.pf, pf[0])
    for d in range(4):
        assert table_ok(got.gc_l[d], gc[1 + d]), d
        assert table_ok(got.pf_l[d], pf[1 + d]), d


def test_oracle_identities():
    """beta_0 = 1, g = beta_1 / 3, Cbak = F11(180) Csca / (4 pi) -- the
    reference's own self-checks (utils/calllmie.c:731-755)."""
    got = libs.run_oracle(example_case())
    assert abs(got.gc[0, 0] - 1.0) < 1e-12
    assert abs(got.scalars["g"] - got.gc[0, 1] / 3.0) < 1e-6
    cbak = got.pf[0, -1] * got.scalars["csca"] / (4 * np.pi)
    assert abs(cbak - got.scalars["cbak"]) / got.scalars["cbak"] < 1e-5


@pytest.mark.skipif(libs.reference() is None, reason="reference library not built here")
@pytest.mark.parametrize("name", ["c1", "gamma", "lognormal_lc", "mono", "nine_derivs"])
def test_oracle_matches_live_reference(name):
    case = all_cases()[name]
    _check(libs.run_oracle(case), libs.run_reference(case, 1), TOL)


def test_fixture_cases_are_current():
    """The fixtures were generated from the case definitions in tests/cases.py."""
    import dataclasses
    import json
    from cases import large_cases
    for name, case in {**all_cases(), **large_cases()}.items():
        with np.load(libs.GOLDEN / f"ref_{name}.npz") as z:
            assert json.loads(str(z["case"])) == json.loads(
                json.dumps(dataclasses.asdict(case), sort_keys=True)), name
