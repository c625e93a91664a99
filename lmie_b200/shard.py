"""Cases over ranks: one process per GPU, no data-path collective.

Polydisperse cases are independent, so N GPUs either solve their own batches
(weak scaling: rank r's batch is generated from seed + r) or split one batch
(strong scaling: contiguous case ranges of balanced estimated cost).  The only
collectives are the timing barrier and the max over ranks of the timed
interval, which bench.py issues through torch.distributed.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

from .abi import Case


def case_cost(case: Case) -> float:
    """Estimated device work of a case: the angular contraction dominates and
    grows as (radii) x (orders) x (angles), with orders and angles both ~ x_max;
    the constant term stands for the per-case launch-independent overhead."""
    x_max = 2.0 * math.pi * case.r2 / case.lam
    n1 = x_max + 4.05 * x_max ** (1.0 / 3.0) + 8.0
    n_r = max(1, case.n_int2) * max(1, case.n_quad)
    return n_r * n1 * 2.0 * n1 * (1.0 + len(case.derivs)) + 1e4


def balanced_ranges(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous [start, end) ranges, one per rank, splitting `costs` at the
    prefix sums nearest to multiples of total / world (every range non-empty
    when there are at least `world` items)."""
    n = len(costs)
    if world < 1:
        raise ValueError("world must be >= 1")
    total = float(sum(costs))
    bounds = [0]
    run, i = 0.0, 0
    for r in range(1, world):
        target = total * r / world
        while i < n and run + costs[i] / 2.0 < target and n - i > world - r:
            run += costs[i]
            i += 1
        i = max(i, bounds[-1] + (1 if n - bounds[-1] > world - r else 0))
        run = float(sum(costs[:i]))
        bounds.append(i)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def strong_slice(cases: Sequence[Case], rank: int, world: int) -> Tuple[int, int]:
    """The case range rank `rank` solves when `world` ranks split `cases`."""
    return balanced_ranges([case_cost(c) for c in cases], world)[rank]


def weak_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s own batch under weak scaling."""
    return seed + rank
