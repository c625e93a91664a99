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


def precision_stress(n_cases: int = 256, seed: int = SEED, n_angles: int = 181) -> List[Case]:
    """Large particles: r_eff uniform in [150, 400] um, v_eff uniform in
    [0.05, 0.2], wavelength uniform in [0.34, 0.55] um, mr uniform in
    [1.31, 1.55], mi log-uniform in [1e-9, 1e-3]; gamma distribution on
    [1e-3 r_eff, r2] with r2 = min(r_eff (1 + 10 v_eff), 5000 lambda / 2 pi), so
    the size parameter reaches at most 5000 (n1 <= 5077, 10154 Gauss angles);
    8000 radii (16 intervals of 500 Gauss points); derivatives w.r.t. mr, mi,
    a1, a2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r_eff = rng.uniform(150.0, 400.0, n_cases)
    v_eff = rng.uniform(0.05, 0.2, n_cases)
    lam = rng.uniform(0.34, 0.55, n_cases)
    mr = rng.uniform(1.31, 1.55, n_cases)
    mi = np.exp(rng.uniform(math.log(1e-9), math.log(1e-3), n_cases))
    cases = []
    for i in range(n_cases):
        r2 = min(r_eff[i] * (1.0 + 10.0 * v_eff[i]), 5000.0 * lam[i] / (2.0 * math.pi))
        cases.append(Case(dist="gamma", lam=float(lam[i]), mr=float(mr[i]), mi=float(mi[i]),
                          a1=float(r_eff[i]), a2=float(v_eff[i]), r1=float(1e-3 * r_eff[i]), r2=float(r2),
                          n_int2=16, n_quad=500, n_angles=n_angles, accuracy=1e-7,
                          derivs=deriv_unit("mr", "mi", "a1", "a2")))
    return cases


class AdjointProblem:
    """Inputs of lmie_solution_adjoint: wavelengths with their refractive
    indices, one binned size distribution and the loss weights."""

    def __init__(self, lam, mr, mi, edges, weight, n_quad, n_angles, c, d11, d12):
        self.lam = np.ascontiguousarray(lam, dtype=np.float64)
        self.mr = np.ascontiguousarray(mr, dtype=np.float64)
        self.mi = np.ascontiguousarray(mi, dtype=np.float64)
        self.edges = np.ascontiguousarray(edges, dtype=np.float64)
        self.weight = np.ascontiguousarray(weight, dtype=np.float64)
        self.n_quad = int(n_quad)
        self.n_angles = int(n_angles)
        self.c = np.ascontiguousarray(c, dtype=np.float64)        # [n_lambda, 3]: c_cext, c_csca, c_g
        self.d11 = np.ascontiguousarray(d11, dtype=np.float64)    # [n_lambda, n_angles]
        self.d12 = np.ascontiguousarray(d12, dtype=np.float64)

    @property
    def n_lambda(self) -> int:
        return len(self.lam)

    @property
    def n_bins(self) -> int:
        return len(self.weight)

    def replace(self, **kw) -> "AdjointProblem":
        a = dict(lam=self.lam, mr=self.mr, mi=self.mi, edges=self.edges, weight=self.weight,
                 n_quad=self.n_quad, n_angles=self.n_angles, c=self.c, d11=self.d11, d12=self.d12)
        a.update(kw)
        return AdjointProblem(**a)


def adjoint_retrieval(n_lambda: int = 256, n_bins: int = 64, n_quad: int = 32, n_angles: int = 181,
                      lam_range=(0.34, 2.25), r_range=(0.02, 20.0), seed: int = SEED) -> AdjointProblem:
    """The retrieval workload: n_lambda wavelengths log-spaced over lam_range
    (um) sharing one distribution of n_bins log-spaced bins over r_range (um)
    with n_quad Gauss points each and seeded bin weights U(0.1, 1); per
    wavelength mr ~ U[1.35, 1.6], mi ~ logU[1e-6, 0.05]; loss weights: c for
    Cext, Csca, g ~ U(-1, 1) scaled to the magnitudes of those outputs, and
    d for P11, P12 at each angle ~ U(-1, 1) / n_angles."""
    rng = np.random.Generator(np.random.PCG64(seed + 5))
    lam = np.exp(np.linspace(math.log(lam_range[0]), math.log(lam_range[1]), n_lambda))
    edges = np.exp(np.linspace(math.log(r_range[0]), math.log(r_range[1]), n_bins + 1))
    weight = rng.uniform(0.1, 1.0, n_bins)
    mr = rng.uniform(1.35, 1.6, n_lambda)
    mi = np.exp(rng.uniform(math.log(1e-6), math.log(0.05), n_lambda))
    c = rng.uniform(-1.0, 1.0, (n_lambda, 3))
    d11 = rng.uniform(-1.0, 1.0, (n_lambda, n_angles)) / n_angles
    d12 = rng.uniform(-1.0, 1.0, (n_lambda, n_angles)) / n_angles
    return AdjointProblem(lam, mr, mi, edges, weight, n_quad, n_angles, c, d11, d12)
