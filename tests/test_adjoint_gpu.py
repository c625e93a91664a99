"""lmie_solution_adjoint on the device against its CPU oracle (per-radius
SIZE_DIST_MONO solves of the oracle with forward-mode mr/mi derivatives,
combined with the bin weights: tests/adjoint_oracle.py) and against central
finite differences of its own loss.

Tolerances: the outputs are FP64 on both sides with different summation
orders (1e-10 relative); at n_max ~ 300 the oracle's phase matrix, taken
from the untruncated expansion whose terms are as large as the forward peak
(at theta = 0 a coherent sum of 2 n_max terms with P_l(1) = 1), carries
about 1e-9 of rounding, so the phase matrix and the loss are compared to
1e-8 there; the mr/mi gradient uses the
closed-form derivative of D_n where the oracle linearises the D_n
recurrence, which agree to the accuracy of the recurrence (1e-8 relative);
central finite differences with Richardson extrapolation over steps of
4e-8 and 2e-8 times max(|p|, 1) (1e-5 relative).
"""
import numpy as np
import pytest

import adjoint_oracle
import lmie_b200
from lmie_b200 import workloads

pytestmark = pytest.mark.gpu


def small(seed=11, r_max=3.0, n_bins=6, n_quad=4, n_angles=19, lam_range=(0.5, 1.1)):
    return workloads.adjoint_retrieval(n_lambda=3, n_bins=n_bins, n_quad=n_quad, n_angles=n_angles,
                                       lam_range=lam_range, r_range=(0.05, r_max), seed=seed)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("r_max,tol", [(3.0, 1e-10), (25.0, 1e-8)])
def test_adjoint_matches_forward_mode(r_max, tol):
    """r_max 25 um at 0.5 um reaches x ~ 300 (n_max ~ 330, six checkpoint
    blocks); there the oracle's phase matrix (an untruncated expansion whose
    terms are as large as the forward peak) carries ~1e-9 of the peak in
    rounding, which bounds the comparison of the outputs and the loss."""
    p = small(r_max=r_max)
    got = lmie_b200.adjoint(p)
    want = adjoint_oracle.solve(p)
    assert abs(got["loss"] - want["loss"]) <= tol * abs(want["loss"]), (got["loss"], want["loss"])
    for name in ("cext", "csca", "g"):
        assert rel(got[name], want[name]) <= 1e-10, (name, rel(got[name], want[name]))
    for name in ("p11", "p12"):
        assert rel(got[name], want[name]) <= tol, (name, rel(got[name], want[name]))
    for name in ("grad_mr", "grad_mi", "grad_weight"):
        assert rel(got[name], want[name]) <= 1e-8, (name, got[name], want[name])


def test_adjoint_full_distribution():
    """The benchmark's distribution -- 64 log-spaced bins x 32 Gauss radii
    over 0.02 - 20 um, 181 angles -- on four wavelengths from 0.34 to
    2.25 um (size parameters up to 370), against the forward-mode oracle
    over all 2048 radii of each wavelength; tolerances as at x ~ 300 above."""
    p = workloads.adjoint_retrieval(n_lambda=4)
    assert p.n_bins == 64 and p.n_quad == 32 and p.n_angles == 181
    got = lmie_b200.adjoint(p)
    want = adjoint_oracle.solve(p, threads=16)
    assert abs(got["loss"] - want["loss"]) <= 1e-8 * abs(want["loss"]), (got["loss"], want["loss"])
    for name in ("cext", "csca", "g"):
        assert rel(got[name], want[name]) <= 1e-10, (name, rel(got[name], want[name]))
    for name in ("p11", "p12", "grad_mr", "grad_mi", "grad_weight"):
        assert rel(got[name], want[name]) <= 1e-8, (name, rel(got[name], want[name]))


def _fd(loss, p, name, idx, rel_h):
    """Central difference with Richardson extrapolation (steps h and h/2):
    weakly absorbing particles of large size parameter have sharp resonances
    in m, so the loss curves strongly on the scale of a 1e-6 relative step."""
    def cd(h):
        v = getattr(p, name)
        up, dn = v.copy(), v.copy()
        up[idx] += h
        dn[idx] -= h
        return (loss(p.replace(**{name: up})) - loss(p.replace(**{name: dn}))) / (2 * h)
    h = rel_h * max(abs(getattr(p, name)[idx]), 1.0)   # mi is small: an absolute step there
    return (4 * cd(h / 2) - cd(h)) / 3


def test_adjoint_finite_differences():
    p = small(seed=12, r_max=10.0)
    base = lmie_b200.adjoint(p)
    loss = lambda q: lmie_b200.adjoint(q)["loss"]
    for k in range(p.n_lambda):
        for name in ("mr", "mi"):
            fd = _fd(loss, p, name, k, 4e-8)
            g = base["grad_" + name][k]
            assert abs(fd - g) <= 1e-5 * max(abs(g), 1e-3), (name, k, fd, g)
    for b in range(0, p.n_bins, 2):
        fd = _fd(loss, p, "weight", b, 4e-8)
        g = base["grad_weight"][b]
        assert abs(fd - g) <= 1e-5 * max(abs(g), 1e-3), (b, fd, g)


def test_adjoint_is_deterministic():
    p = small(seed=13)
    a, b = lmie_b200.adjoint(p), lmie_b200.adjoint(p)
    assert a["loss"] == b["loss"]
    assert np.array_equal(a["grad_mr"], b["grad_mr"]) and np.array_equal(a["grad_weight"], b["grad_weight"])


def test_adjoint_rejects_bad_input():
    p = small()
    with pytest.raises(RuntimeError):
        lmie_b200.adjoint(p.replace(edges=p.edges[::-1].copy()))
    with pytest.raises(RuntimeError):
        lmie_b200.adjoint(p.replace(n_angles=1, d11=p.d11[:, :1].copy(), d12=p.d12[:, :1].copy()))
