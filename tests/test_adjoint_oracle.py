"""The adjoint's CPU oracle against central finite differences of itself
(no GPU): pins the combination formulas and the chain rule of
tests/adjoint_oracle.py before it is used as the reference of the device
adjoint."""
import numpy as np
import pytest

import adjoint_oracle
from lmie_b200 import workloads


def tiny(seed=3):
    return workloads.adjoint_retrieval(n_lambda=2, n_bins=3, n_quad=3, n_angles=7, lam_range=(0.5, 0.9),
                                       r_range=(0.1, 3.0), seed=seed)


def test_oracle_gradient_matches_finite_differences():
    p = tiny()
    base = adjoint_oracle.solve(p)
    for k in range(p.n_lambda):
        for name in ("mr", "mi"):
            v = getattr(p, name).copy()
            h = 1e-6 * v[k]
            up, dn = v.copy(), v.copy()
            up[k] += h
            dn[k] -= h
            fd = (adjoint_oracle.solve(p.replace(**{name: up}))["loss"] -
                  adjoint_oracle.solve(p.replace(**{name: dn}))["loss"]) / (2 * h)
            g = base["grad_" + name][k]
            assert abs(fd - g) <= 1e-6 * max(abs(g), 1e-8 * abs(base["loss"]) / h), (name, k, fd, g)
    for b in range(p.n_bins):
        w = p.weight.copy()
        h = 1e-6 * w[b]
        up, dn = w.copy(), w.copy()
        up[b] += h
        dn[b] -= h
        fd = (adjoint_oracle.solve(p.replace(weight=up))["loss"] -
              adjoint_oracle.solve(p.replace(weight=dn))["loss"]) / (2 * h)
        g = base["grad_weight"][b]
        assert abs(fd - g) <= 1e-6 * max(abs(g), 1e-3), (b, fd, g)


def test_oracle_outputs_are_consistent():
    p = tiny(seed=4)
    o = adjoint_oracle.solve(p)
    assert np.all(o["cext"] > 0) and np.all(o["csca"] > 0) and np.all(o["csca"] <= o["cext"] * (1 + 1e-12))
    assert np.all(np.abs(o["g"]) < 1)
    assert np.all(o["p11"] > 0)
