"""Named polydisperse cases shared by the fixture generator and the tests.

The sizes follow the reference's own example (examples/example_c.c:44-110)
and the workloads the benchmark is quoted on; the edge cases cover every
size distribution, every kind of derivative input, both expansion kinds,
save_control and the odd/even Gauss-point paths.
"""
from __future__ import annotations

import math
from typing import Dict, List

from lmie_b200.abi import Case, deriv_unit

ALL_DERIVS = [{"lambda": 1.0}, {"mr": 1.0}, {"mi": 1.0}, {"a1": 1.0}, {"a2": 1.0}, {"a3": 1.0},
              {"a4": 1.0}, {"a5": 1.0}, {"r1": 1.0}, {"r2": 1.0}, {"mr": 0.5, "a1": 2.0}]


def example_case() -> Case:
    """The reference's example: accumulation-mode mineral dust at 2.25 um."""
    return Case(dist="log_normal", lam=2.25, mr=1.53, mi=0.0054, a1=0.39, a2=0.4805,
                r1=0.005, r2=50.0, n_int2=64, n_quad=64, n_angles=181, accuracy=1e-7,
                derivs=deriv_unit("mr", "mi", "a1", "a2"))


def c1_case(accuracy: float = 1e-7) -> Case:
    """Plain FP64 solve: lognormal r_g = 0.1 um, sigma_g = 1.5, 200 radii, 0.55 um."""
    return Case(dist="log_normal", lam=0.55, mr=1.45, mi=1e-3, a1=0.1,
                a2=math.log(1.5) ** 2, r1=0.005, r2=2.0, n_int2=1, n_quad=200,
                n_angles=181, accuracy=accuracy)


def c2_case() -> Case:
    """Forward-linearized cloud droplet: gamma r_eff = 10 um, v_eff = 0.1,
    r in [0.01, 60] um, 4 x 500 radii, 0.865 um, m = 1.335 + 1e-6 i,
    derivatives w.r.t. mr, mi, r_eff, v_eff."""
    return Case(dist="gamma", lam=0.865, mr=1.335, mi=1e-6, a1=10.0, a2=0.1, r1=0.01,
                r2=60.0, n_int2=4, n_quad=500, n_angles=181, accuracy=1e-7,
                derivs=deriv_unit("mr", "mi", "a1", "a2"))


def small_cases() -> Dict[str, Case]:
    """Cases the CPU oracle finishes in well under a second each."""
    d = ALL_DERIVS
    return {
        "c1": c1_case(),
        "c1_acc0": c1_case(0.0),
        "mgamma": Case(dist="modified_gamma", lam=0.6, a1=2.0, a2=0.5, a3=1.0, r1=0.01, r2=3.0,
                       n_int2=2, n_quad=50, derivs=d),
        "lognormal_lc": Case(dist="log_normal", lam=0.6, a1=0.3, a2=0.3, r1=0.01, r2=3.0,
                             n_int2=2, n_quad=50, calc_gc=0, calc_lc=1, derivs=d),
        "lognormal_gc_lc": Case(dist="log_normal", lam=0.6, a1=0.3, a2=0.3, r1=0.01, r2=3.0,
                                n_int2=2, n_quad=50, calc_gc=1, calc_lc=1, derivs=d),
        "power_law": Case(dist="power_law", lam=0.6, a1=0.5, a2=0.2, n_int2=3, n_quad=40,
                          derivs=d),
        "gamma": Case(dist="gamma", lam=0.6, a1=0.5, a2=0.2, r1=0.01, r2=4.0, n_int2=3,
                      n_quad=40, derivs=d),
        "mod_power_law": Case(dist="modified_power_law", lam=0.6, a1=-3.0, r1=0.1, r2=2.0,
                              n_int1=2, n_int2=3, n_quad=30, derivs=d),
        "bimodal": Case(dist="modified_bimodal_log_normal", lam=0.6, a1=0.2, a2=0.2, a3=1.0,
                        a4=0.3, a5=0.1, r1=0.01, r2=4.0, n_int2=3, n_quad=40, derivs=d),
        "exponential": Case(dist="exponential", lam=0.6, a1=2.0, r1=0.01, r2=2.0, n_int2=3,
                            n_quad=40),
        "mono": Case(dist="mono", lam=0.6, a1=1.3, r1=1.3, r2=1.3, derivs=d),
        "no_angles": Case(dist="gamma", lam=0.6, a1=0.5, a2=0.2, r1=0.01, r2=4.0, n_int2=3,
                          n_quad=40, calc_gc=0, calc_pf=0, derivs=d),
        "odd_quad": Case(dist="gamma", lam=0.6, a1=0.5, a2=0.2, r1=0.01, r2=4.0, n_int2=3,
                         n_quad=41, n_angles=19, derivs=d),
        "tiny_x": Case(dist="log_normal", lam=10.0, a1=0.01, a2=0.2, r1=0.001, r2=0.05,
                       n_int2=1, n_quad=16, n_angles=7, derivs=deriv_unit("mr", "mi", "lambda")),
        "absorbing": Case(dist="gamma", lam=0.5, mr=1.75, mi=0.5, a1=1.0, a2=0.2, r1=0.05,
                          r2=6.0, n_int2=2, n_quad=60, derivs=deriv_unit("mr", "mi", "r2")),
        "nine_derivs": Case(dist="modified_bimodal_log_normal", lam=0.7,
                            a1=0.2, a2=0.2, a3=1.0, a4=0.3, a5=0.1, r1=0.01, r2=3.0, n_int2=2,
                            n_quad=40, derivs=[{"mr": 1.0}, {"mi": 1.0}, {"lambda": 1.0},
                                               {"r1": 1.0}, {"r2": 1.0}, {"mr": 2.0, "mi": 1.0},
                                               {"a1": 1.0}, {"a2": 1.0}, {"a3": 1.0}]),
        "save1": Case(dist="gamma", lam=0.6, a1=0.5, a2=0.2, r1=0.01, r2=4.0, n_int2=2,
                      n_quad=20, save_control=1, derivs=deriv_unit("a1", "a2")),
    }


def medium_cases() -> Dict[str, Case]:
    """Cases that take the CPU oracle a few seconds."""
    return {
        "example": example_case(),
        "c2": c2_case(),
        "large_x_cross_sections": Case(dist="gamma", lam=0.5, mr=1.33, mi=1e-4, a1=300.0,
                                       a2=0.1, r1=350.0, r2=398.0, n_int2=1, n_quad=12,
                                       calc_gc=0, calc_pf=0, derivs=deriv_unit("mr", "mi")),
        "x1000_few_radii": Case(dist="gamma", lam=0.5, mr=1.50, mi=1e-3, a1=60.0, a2=0.05,
                                r1=70.0, r2=80.0, n_int2=1, n_quad=8, n_angles=91,
                                derivs=deriv_unit("mr", "a1")),
    }


def all_cases() -> Dict[str, Case]:
    d = dict(small_cases())
    d.update(medium_cases())
    return d


# cases of the seeded 4096-case uneven workload (workloads.batched_uneven)
# whose largest size parameter is above 500, spread over 502 .. 1063
UNEVEN_LARGE_X = (3278, 1168, 4034, 2007, 2343, 2904, 517, 2963)


def large_cases() -> Dict[str, Case]:
    """Cases at the sizes the benchmark runs, pinned to the reference's own
    outputs (seconds of reference CPU time each): the large-particle
    configuration with every output (size parameter up to 5000, n1 = 5077,
    10154 Gauss angles, n_coef ~ 10^4; 8 radii instead of 8000, since each
    radius' work is the same) and eight cases of the uneven workload with
    size parameters from 502 to 1063."""
    from lmie_b200 import workloads
    d = {"x5000_full": Case(dist="gamma", lam=0.5, mr=1.33, mi=1e-4, a1=300.0, a2=0.1, r1=350.0,
                            r2=398.0, n_int2=1, n_quad=8, n_angles=181, accuracy=1e-7,
                            derivs=deriv_unit("mr", "mi", "a1", "a2"))}
    uneven = workloads.batched_uneven(4096)
    for i in UNEVEN_LARGE_X:
        d[f"uneven_{i}"] = uneven[i]
    return d


def case_names() -> List[str]:
    return list(all_cases().keys())
