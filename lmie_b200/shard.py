"""Work over ranks, one process per GPU.

Cases: polydisperse cases are independent, so N GPUs either solve their own
batches (weak scaling: rank r's batch is generated from seed + r) or split
one batch (strong scaling: contiguous case ranges of balanced estimated
cost), with no data-path collective; the only collectives are the timing
barrier and the max over ranks of the timed interval, which bench.py issues
through torch.distributed.

Radii: one large case can be shared by a group of GPUs (the reference's
use_mpi, src/lmie_schedule.c:459-921): each rank solves its share of the
radii, one FP64 all-reduce sums the integrals, and every rank finishes.  The
library sums either with its own NCCL all-reduce on the solve's stream
(`use_nccl_group`) or through a callback (`use_torch_group`, torch.distributed).
"""
from __future__ import annotations

import ctypes as C
import math
import sys
from typing import List, Sequence, Tuple

from .abi import Case, REDUCE_FN


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


# ---- radius sharing --------------------------------------------------------

class _DeviceDoubles:
    """`count` doubles at a device address, as torch sees them through the
    CUDA array interface (no copy)."""

    def __init__(self, addr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (addr, False),
                                         "version": 3, "strides": None}


def device_doubles(addr: int, count: int):
    import torch
    return torch.as_tensor(_DeviceDoubles(addr, count), device="cuda")


def torch_reducer(group=None, wrap=device_doubles):
    """A lmieb_reduce_fn that sums the library's integrals over the
    torch.distributed `group` (all_reduce, SUM) and returns once the sum is in
    place.  `wrap(address, count)` turns the buffer into a tensor: device
    memory by default; tests on CPU ranks pass a host wrapper."""
    import torch
    import torch.distributed as dist

    def fn(buf, count, stream, ctx):
        try:
            t = wrap(C.cast(buf, C.c_void_p).value, int(count))
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            if t.is_cuda:
                torch.cuda.synchronize(t.device)
            return 0
        except Exception as e:  # reported to the library as a failed reduction
            print(f"ERROR: lmie_b200 radius-group reduction: {e}", file=sys.stderr)
            return -1

    return REDUCE_FN(fn)


def use_torch_group(lib, group=None):
    """Makes the library share the radii of lmie_solution(..., use_mpi=1)
    calls with the ranks of the torch.distributed `group`.  Returns the
    callback object, which must stay alive while it is registered."""
    import torch.distributed as dist
    cb = torch_reducer(group)
    if lib.lmieb_set_radius_group(dist.get_rank(group), dist.get_world_size(group), cb, None) != 0:
        raise RuntimeError("lmieb_set_radius_group failed")
    return cb


def use_nccl_group(lib, group=None) -> None:
    """The same with the library's own NCCL all-reduce (no host round trip):
    rank 0 of `group` creates the NCCL id, the group's collective sends it to
    the others, and every rank joins the communicator."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    uid = (C.c_char * 128)()
    ok = rank != 0 or lib.lmieb_nccl_unique_id(uid) == 0
    obj = [bytes(uid) if ok else b""] if rank == 0 else [None]
    src = 0 if group is None else dist.get_global_rank(group, 0)
    dist.broadcast_object_list(obj, src=src, group=group)
    if len(obj[0]) != 128:
        raise RuntimeError("lmieb_nccl_unique_id failed on rank 0")
    uid = (C.c_char * 128).from_buffer_copy(obj[0])
    if lib.lmieb_set_radius_group_nccl(uid, rank, world) != 0:
        raise RuntimeError("lmieb_set_radius_group_nccl failed")


def leave_group(lib) -> None:
    """Ends radius sharing: use_mpi calls solve every radius here again."""
    if lib.lmieb_set_radius_group(0, 1, REDUCE_FN(), None) != 0:
        raise RuntimeError("lmieb_set_radius_group failed")
