"""Radius sharing over a group of GPUs: the B200 form of the reference's
use_mpi (src/lmie_schedule.c:459-921, 1125-1152), where the MPI master deals
the radii of one solve out to worker ranks and adds up their cross sections
and phase-matrix integrals before normalising.

Every GPU run here has one GPU, so the group is exercised in the forms one GPU
allows, each against the reference's own outputs (golden fixtures) or the
whole solve:
  * the two-call form: the integrals of world = 2 or 3 shares, summed on the
    host and finished, match the reference to the parity bar 1e-10 (only the
    order of the radius sums differs from the whole solve);
  * a share with no radii (more ranks than radii) contributes zeros;
  * the in-call form as rank 0 of a world of 2, whose reduction callback adds
    rank 1's integrals to the device buffer -- the sum an all-reduce makes;
  * the in-call form with a one-rank group, through a callback and through
    the library's own NCCL all-reduce: bit-identical to the whole solve.
The CPU tests cover the host side: the integral count, argument checks, and
the torch.distributed callback across two gloo ranks.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest

import libs
from cases import all_cases
from lmie_b200 import abi, shard

TOL = 1e-10


def _lib():
    lib = libs.product()
    abi.bind_group(lib)
    return lib


def _assert_close(got, want, tol=TOL, label=""):
    assert got.rc == 0, label
    err = libs.compare(got, want)
    assert err["n_coef"] <= 1, (label, got.n_coef, want.n_coef)
    bad = {k: v for k, v in err.items() if k != "n_coef" and v > tol}
    assert not bad, (label, bad)


def _assert_identical(got, want):
    assert got.rc == 0 and got.n_coef == want.n_coef
    assert got.scalars == want.scalars
    for k, v in want.scalars_l.items():
        assert np.array_equal(got.scalars_l[k], v), k
    for name in ("gc", "lc", "pf", "gc_l", "lc_l", "pf_l"):
        w = getattr(want, name)
        if w is not None:
            assert np.array_equal(getattr(got, name), w), name


# ---- CPU --------------------------------------------------------------------

def test_partial_size_counts_the_integrals():
    lib = _lib()
    for name in ("c2", "no_angles", "nine_derivs", "power_law"):
        case = all_cases()[name]
        blk = abi.InputBlock(case)
        nq = 0
        if case.calc_gc or case.calc_lc:
            nq = lib.lmie_calc_max_coef(case.lam, blk.s.dist_type, case.a1, case.a2, case.a3, case.r1, case.r2)
        assert lib.lmieb_partial_size(C.byref(blk.s)) == 4 * (1 + case.n_derivs) * (1 + nq), name


def test_group_arguments_are_checked():
    lib = _lib()
    rank, world = C.c_int(-1), C.c_int(-1)
    assert lib.lmieb_get_radius_group(C.byref(rank), C.byref(world)) == 0
    assert (rank.value, world.value) == (0, 1)
    null = abi.REDUCE_FN()
    assert lib.lmieb_set_radius_group(0, 2, null, None) == -1        # world > 1 needs a reduction
    assert lib.lmieb_set_radius_group(2, 2, null, None) == -1        # rank outside the group
    assert lib.lmieb_set_radius_group(0, 0, null, None) == -1
    keep = abi.REDUCE_FN(lambda buf, count, stream, ctx: 0)
    assert lib.lmieb_set_radius_group(1, 3, keep, None) == 0
    assert lib.lmieb_get_radius_group(C.byref(rank), C.byref(world)) == 1
    assert (rank.value, world.value) == (1, 3)
    shard.leave_group(lib)
    assert lib.lmieb_get_radius_group(C.byref(rank), C.byref(world)) == 0
    assert (rank.value, world.value) == (0, 1)


def test_sharing_rejects_save_control_before_any_device_work():
    lib = _lib()
    case = all_cases()["save1"]
    blk = abi.InputBlock(case)
    acc = np.zeros(lib.lmieb_partial_size(C.byref(blk.s)))
    assert lib.lmieb_solution_partial(C.byref(blk.s), 0, 2, acc.ctypes.data_as(abi.PD), 0) == -1
    assert lib.lmieb_solution_partial(C.byref(blk.s), 2, 2, acc.ctypes.data_as(abi.PD), 0) == -1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _host_doubles(addr, count):
    import torch
    return torch.from_numpy(np.ctypeslib.as_array(C.cast(addr, abi.PD), shape=(count,)))


def _gloo_rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cb = shard.torch_reducer(wrap=_host_doubles)
        buf = np.arange(7, dtype=np.float64) * (rank + 1) + 0.25 * rank
        rc = cb(buf.ctypes.data_as(abi.PD), buf.size, None, None)
        q.put((rank, rc, buf.copy()))
    finally:
        dist.destroy_process_group()


def test_torch_reducer_sums_over_two_gloo_ranks():
    """The callback the library calls with its integrals, on two CPU ranks:
    every rank ends with the sum, in place."""
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.arange(7, dtype=np.float64) * 3 + 0.25
    for rank, rc, buf in res:
        assert rc == 0
        assert np.array_equal(buf, want), rank


# ---- GPU --------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name, world", [("c2", 2), ("gamma", 3), ("nine_derivs", 2),
                                         ("lognormal_gc_lc", 3), ("no_angles", 2), ("example", 4),
                                         ("mono", 2)])
def test_shares_summed_on_the_host_match_the_reference(name, world):
    lib = _lib()
    case = all_cases()[name]
    parts = [abi.solve_partial(lib, case, r, world) for r in range(world)]
    if name == "mono":
        assert not parts[1].any()       # one radius: rank 1's share is empty
    got = abi.solve_finish(lib, case, np.sum(parts, axis=0))
    _assert_close(got, libs.golden(name), label=name)
    _assert_close(got, libs.run_product(case), label=name)


@pytest.mark.gpu
def test_group_callback_as_rank_0_of_two():
    """lmie_solution(..., use_mpi=1) as rank 0 of two: the callback adds rank
    1's integrals (two-call form) to the device buffer, as an all-reduce over
    two GPUs would."""
    import torch
    lib = _lib()
    case = all_cases()["c2"]
    other = abi.solve_partial(lib, case, 1, 2)
    seen = []

    def add_rank1(buf, count, stream, ctx):
        # the integrals, then the group's failure count (rank 1 did not fail)
        t = shard.device_doubles(C.cast(buf, C.c_void_p).value, int(count))
        t[:other.size].add_(torch.from_numpy(other).to(t.device))
        torch.cuda.synchronize(t.device)
        seen.append(int(count))
        return 0

    cb = abi.REDUCE_FN(add_rank1)
    assert lib.lmieb_set_radius_group(0, 2, cb, None) == 0
    try:
        got = abi.solve(lib, case, use_mpi=1)
    finally:
        shard.leave_group(lib)
    assert seen == [other.size + 1]
    _assert_close(got, libs.golden("c2"), label="c2")
    # without use_mpi the group is not used
    assert lib.lmieb_set_radius_group(0, 2, cb, None) == 0
    try:
        whole = abi.solve(lib, case, use_mpi=0)
    finally:
        shard.leave_group(lib)
    assert seen == [other.size + 1]
    _assert_identical(whole, libs.run_product(case))


@pytest.mark.gpu
@pytest.mark.parametrize("site", ["prepare", "alloc", "h2d"])
def test_group_failure_is_shared(site):
    """A process whose solve fails before the group's sum -- on the host
    (preparation) or on the device side (arena, upload; injected by
    LMIEB_FAULT) -- still takes part in the sum, once, with zero integrals
    and a failure count of 1, so no process is left waiting; a healthy
    process whose sum carries a peer's failure returns -1 as well; and the
    group works again afterwards."""
    import os
    import torch
    lib = _lib()
    case = all_cases()["c2"]
    n = abi.solve_partial(lib, case, 1, 2).size          # the integrals
    calls = []

    def record(buf, count, stream, ctx):
        t = shard.device_doubles(C.cast(buf, C.c_void_p).value, int(count))
        torch.cuda.synchronize(t.device)
        calls.append((int(count), float(t[-1]), float(t[:-1].abs().sum())))
        return 0

    cb = abi.REDUCE_FN(record)
    assert lib.lmieb_set_radius_group(1, 2, cb, None) == 0
    try:
        os.environ["LMIEB_FAULT"] = site
        try:
            failed = abi.solve(lib, case, use_mpi=1)
        finally:
            os.environ.pop("LMIEB_FAULT", None)
        assert failed.rc == -1
        assert calls == [(n + 1, 1.0, 0.0)], calls
    finally:
        shard.leave_group(lib)

    # a healthy rank 0 whose peer failed: the peer's block is zeros and a 1
    def peer_failed(buf, count, stream, ctx):
        t = shard.device_doubles(C.cast(buf, C.c_void_p).value, int(count))
        t[-1] += 1.0
        torch.cuda.synchronize(t.device)
        return 0

    cb2 = abi.REDUCE_FN(peer_failed)
    assert lib.lmieb_set_radius_group(0, 2, cb2, None) == 0
    try:
        assert abi.solve(lib, case, use_mpi=1).rc == -1
    finally:
        shard.leave_group(lib)
    # and the library keeps working
    _assert_identical(abi.solve(lib, case), libs.run_product(case))


@pytest.mark.gpu
def test_group_of_one_is_the_whole_solve():
    lib = _lib()
    case = all_cases()["nine_derivs"]
    want = libs.run_product(case)
    cb = abi.REDUCE_FN(lambda buf, count, stream, ctx: 0)
    assert lib.lmieb_set_radius_group(0, 1, cb, None) == 0
    try:
        got = abi.solve(lib, case, use_mpi=1)
    finally:
        shard.leave_group(lib)
    _assert_identical(got, want)


@pytest.mark.gpu
def test_nccl_group_of_one_is_the_whole_solve():
    """The library's own NCCL all-reduce, queued on the solve's stream, with a
    one-rank communicator."""
    import torch  # noqa: F401  (the process's libnccl.so.2, as in a torch program)
    lib = _lib()
    case = all_cases()["c2"]
    want = libs.run_product(case)
    uid = (C.c_char * 128)()
    assert lib.lmieb_nccl_unique_id(uid) == 0
    assert lib.lmieb_set_radius_group_nccl(uid, 0, 1) == 0
    try:
        rank, world = C.c_int(), C.c_int()
        assert lib.lmieb_get_radius_group(C.byref(rank), C.byref(world)) == 1
        assert (rank.value, world.value) == (0, 1)
        got = abi.solve(lib, case, use_mpi=1)
    finally:
        shard.leave_group(lib)
    _assert_identical(got, want)

