"""lmie_cross_sections_noalloc: the entry point for callers that cannot
allocate device memory (their memory pool owns the GPU, or they cannot pay
cudaMalloc's device-wide synchronisation).  It is called through the C ABI on
buffers the test owns, and its output must match what lmie_solution returns
for a single-radius distribution, within the parity tolerance of the other
tests, on two calls in a row (the second call reuses the shared scratch)."""
import ctypes as C

import numpy as np
import pytest

import libs
from lmie_b200 import abi

pytestmark = pytest.mark.gpu

TOL = 1e-10
NAMES = ("cext", "csca", "cbak", "g")


def _lib():
    lib = libs.product()
    f = lib.lmie_cross_sections_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                  C.c_void_p]
    return lib


def _via_solution(lam, mr, mi, radii):
    out = np.zeros((4, len(radii)))
    for i, r in enumerate(radii):
        res = libs.run_product(abi.Case(dist="mono", lam=lam, mr=mr, mi=mi, a1=float(r),
                                        r1=float(r), r2=float(r), calc_gc=0, calc_pf=0))
        assert res.rc == 0
        out[:, i] = [res.scalars[k] for k in NAMES]
    return out


def _via_noalloc(lib, lam, mr, mi, radii):
    import torch
    d_r = torch.tensor(np.asarray(radii, dtype=np.float64), device="cuda")
    d_out = torch.full((4, len(radii)), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.lmie_cross_sections_noalloc(len(radii), d_r.data_ptr(), lam, mr, mi,
                                         d_out.data_ptr(), None)
    assert rc == 0
    return d_out.cpu().numpy()


def test_noalloc_matches_lmie_solution_on_two_calls():
    lib = _lib()
    calls = [
        (0.6, 1.45, 1e-2, np.geomspace(0.01, 60.0, 48)),      # x up to ~628
        (0.45, 1.33, 1e-5, np.linspace(0.5, 20.0, 33)),       # fewer radii, new index
    ]
    for lam, mr, mi, radii in calls:
        got = _via_noalloc(lib, lam, mr, mi, radii)
        want = _via_solution(lam, mr, mi, radii)
        for q, name in enumerate(NAMES):
            assert libs.relmax(got[q], want[q]) < TOL, (lam, name)


def test_noalloc_dense_size_parameters():
    """Size parameters packed densely over (0, 900], 1024 radii per call: the
    truncation orders are the host's at every one of them, so the results
    are lmie_solution's (one batch call of SIZE_DIST_MONO cases)."""
    lib = _lib()
    lam, mr, mi = 0.55, 1.38, 3e-4
    x = np.concatenate([np.geomspace(1e-3, 900.0, 1024), np.linspace(0.45, 900.0, 1024)])
    radii = x * lam / (2.0 * np.pi)
    cases = [abi.Case(dist="mono", lam=lam, mr=mr, mi=mi, a1=float(r), r1=float(r), r2=float(r),
                      calc_gc=0, calc_pf=0) for r in radii]
    res = abi.solve_batch(libs.product(), cases, n_threads=8)
    want = np.array([[r.scalars[k] for r in res] for k in NAMES])
    assert all(r.rc == 0 for r in res)
    for part in (slice(0, 1024), slice(1024, 2048)):
        got = _via_noalloc(lib, lam, mr, mi, radii[part])
        for q, name in enumerate(NAMES):
            assert libs.relmax(got[q], want[q, part]) < TOL, name


def test_noalloc_rejects_requests_beyond_its_limits():
    import torch
    lib = _lib()
    d_r = torch.full((1025,), 1.0, dtype=torch.float64, device="cuda")
    d_out = torch.zeros((4, 1025), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert lib.lmie_cross_sections_noalloc(1025, d_r.data_ptr(), 0.5, 1.4, 0.0,
                                           d_out.data_ptr(), None) == -1
    # a radius with size parameter above 900 is refused by the kernel's own check
    d_r = torch.tensor([1.0, 100.0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert lib.lmie_cross_sections_noalloc(2, d_r.data_ptr(), 0.5, 1.4, 0.0,
                                           d_out.data_ptr(), None) == -1
    # and the entry point still works afterwards
    got = _via_noalloc(lib, 0.5, 1.4, 1e-3, [0.3, 1.0])
    want = _via_solution(0.5, 1.4, 1e-3, [0.3, 1.0])
    assert libs.relmax(got, want) < TOL
