"""Seeded synthetic workloads of the benchmark configurations.

Inputs only -- shapes, sizes and value distributions of the configurations the
benchmark is quoted on; nothing is read from disk.  All generators use numpy's
PCG64 with a fixed default seed.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .abi import Case, deriv_unit

SEED = 20261203


def batched_uneven(n_cases: int = 4096, seed: int = SEED, n_angles: int = 181) -> List[Case]:
    """Independent cases of uneven size: r_eff log-uniform in [0.05, 20] um,
    v_eff uniform in [0.02, 0.3], wavelength uniform in [0.34, 2.1] um,
    mr uniform in [1.33, 1.60], mi log-uniform in [1e-8, 0.1]; gamma or
    log-normal distribution 50/50; r in [1e-3 r_eff, r_eff (1 + 10 v_eff)];
    radii 100 per 100 units of size parameter (100..2000) as intervals of 100
    Gauss points; derivatives w.r.t. mr, mi, a1, a2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r_eff = np.exp(rng.uniform(math.log(0.05), math.log(20.0), n_cases))
    v_eff = rng.uniform(0.02, 0.3, n_cases)
    lam = rng.uniform(0.34, 2.1, n_cases)
    mr = rng.uniform(1.33, 1.60, n_cases)
    mi = np.exp(rng.uniform(math.log(1e-8), math.log(0.1), n_cases))
    kind = rng.uniform(0.0, 1.0, n_cases) < 0.5
    cases = []
    for i in range(n_cases):
        r2 = r_eff[i] * (1.0 + 10.0 * v_eff[i])
        r1 = 1e-3 * r_eff[i]
        x_max = 2.0 * math.pi * r2 / lam[i]
        n_r = int(min(max(100 * math.ceil((x_max + 20.0) / 100.0), 100), 2000))
        if kind[i]:
            dist, a1, a2 = "gamma", r_eff[i], v_eff[i]
        else:
            dist = "log_normal"
            a2 = math.log(1.0 + v_eff[i])
            a1 = r_eff[i] / (1.0 + v_eff[i]) ** 2.5
        cases.append(Case(dist=dist, lam=float(lam[i]), mr=float(mr[i]), mi=float(mi[i]),
                          a1=float(a1), a2=float(a2), r1=float(r1), r2=float(r2),
                          n_int2=n_r // 100, n_quad=100, n_angles=n_angles, accuracy=1e-7,
                          derivs=deriv_unit("mr", "mi", "a1", "a2")))
    return cases
